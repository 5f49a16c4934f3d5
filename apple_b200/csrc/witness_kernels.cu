// Witness columns -> Circle FFT-basis coefficients on the device
// (CircleWitnessToFFTBasisPlanV1, CircleWitnessFFTBasis.swift:226-590; the
// transform is CircleWitnessToFFTBasisOracleV1.transformMonomialColumns, i.e.
// CircleCodeword.swift:187-263 for each column).
//
// The reference multiplies by a dense n x n M31 matrix whose column k is the line
// basis of x^k (built on the CPU, tiled past 4096 columns).  That matrix factors as
// L * B: B takes monomials to Chebyshev coefficients, L takes Chebyshev
// coefficients to the line basis.  B has a closed form,
//   x^k = 2^(1-k) * sum_j C(k, j) T_(k-2j)        (the T_0 term halved),
// so with a_k = x_k * 2^(1-k) * k! the Chebyshev coefficient of T_m is
//   c_m = sum_j a_(m+2j) / (j! (m+j)!)            (halved for m = 0),
// computed here from factorial tables without storing any matrix: each term is
// one M31 product of two table entries and a QM31-by-M31 product.  L is the
// reference's split recursion (low[i] -= high[half-i]/2 after doubling the high
// half), run level by level: the pair (i, s-i) of a block of size s becomes
// (c_i - c_(s-i), 2 c_(s-i)).
#include "azk_field.cuh"
#include "azk_internal.h"

namespace azk {

// 2^e mod p for e in [0, 31): the value 1 shifted left by e (2^31 = 1 mod p).
__device__ __forceinline__ uint32_t pow2_m31(uint32_t e) { return 1u << (e % 31); }

// fact[k] = k! mod p, prefix products of max(k, 1) over one 1024-element segment
// per block; seg[b] = the segment's product.
__global__ void __launch_bounds__(1024) fact_segments_kernel(uint32_t* __restrict__ fact, uint32_t* __restrict__ seg, uint64_t n) {
  __shared__ uint32_t wsum[32];
  const uint64_t k = (uint64_t)blockIdx.x * 1024 + threadIdx.x;
  uint32_t v = k < n ? (k == 0 ? 1u : (uint32_t)k) : 1u;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (uint32_t)o) v = m31_mul(v, u);
  }
  if (lane == 31) wsum[warp] = v;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t u = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= (uint32_t)o) w = m31_mul(w, u);
    }
    wsum[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v = m31_mul(v, wsum[warp - 1]);
  if (k < n) fact[k] = v;
  if (threadIdx.x == 1023) seg[blockIdx.x] = v;
}

// Exclusive prefix products of the segment products (one thread: a few thousand
// multiplies, once per plan).
__global__ void fact_seg_prefix_kernel(uint32_t* __restrict__ seg, uint32_t nseg) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t run = 1;
  for (uint32_t b = 0; b < nseg; b++) {
    uint32_t v = seg[b];
    seg[b] = run;
    run = m31_mul(run, v);
  }
}

// fact[k] *= prefix of its segment; ifact[k] = 1 / k!; scale[k] = 2^(1-k) k!.
__global__ void fact_finish_kernel(uint32_t* __restrict__ fact, const uint32_t* __restrict__ seg, uint32_t* __restrict__ ifact,
                                   uint32_t* __restrict__ scale, uint64_t n) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const uint32_t f = m31_mul(fact[k], seg[k >> 10]);
  fact[k] = f;
  ifact[k] = m31_inv(f);
  // 2^(1-k) = 2^((1 - k) mod 31)
  const uint32_t e = (uint32_t)((1 + 31 * ((k / 31) + 1) - k) % 31);
  scale[k] = m31_mul(f, pow2_m31(e));
}

// a[k] = column[k] * scale[k] for k < count (QM31 by M31), zero up to capacity.
__global__ void witness_scale_kernel(const uint4* __restrict__ col, uint64_t count, const uint32_t* __restrict__ scale, uint4* __restrict__ a,
                                     uint64_t capacity) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= capacity) return;
  if (k < count) {
    const uint4 v = col[k];
    const qm31 r = q_mul_m31(qm31{v.x, v.y, v.z, v.w}, scale[k]);
    a[k] = make_uint4(r.a, r.b, r.c, r.d);
  } else {
    a[k] = make_uint4(0u, 0u, 0u, 0u);
  }
}

// Chebyshev coefficients of both columns: one output index m per thread, the
// sum over j in chunks whose table entries and scaled coefficients are staged in
// shared memory.  blockIdx.y takes a slice of the j range (so short outputs still
// fill the GPU) and writes its partial sums; chebyshev_sum_kernel adds the slices.
static constexpr uint32_t kChebM = 256;  // outputs per block
static constexpr uint32_t kChebJ = 256;  // terms per chunk
static constexpr uint32_t kWitnessBlockTarget = 296;  // two blocks per SM

__global__ void __launch_bounds__(kChebM) chebyshev_kernel(const uint4* __restrict__ ax, const uint4* __restrict__ ay, uint64_t count,
                                                          const uint32_t* __restrict__ ifact, uint4* __restrict__ px, uint4* __restrict__ py,
                                                          uint64_t capacity, uint64_t chunks_per_slice) {
  __shared__ uint32_t s_ij[kChebJ];            // ifact[j0 + t]
  __shared__ uint32_t s_imj[kChebM + kChebJ];  // ifact[m0 + j0 + t]
  __shared__ uint4 s_ax[kChebM + 2 * kChebJ];  // a[m0 + 2 j0 + t]
  __shared__ uint4 s_ay[kChebM + 2 * kChebJ];
  const uint64_t m0 = (uint64_t)blockIdx.x * kChebM;
  const uint64_t m = m0 + threadIdx.x;
  qm31 sx = {0, 0, 0, 0}, sy = {0, 0, 0, 0};
  // terms need m + 2j < count: j < (count - m0 + 1) / 2 for the block's first m
  const uint64_t jend = count > m0 ? (count - m0 + 1) / 2 : 0;
  const uint64_t jlo = (uint64_t)blockIdx.y * chunks_per_slice * kChebJ;
  const uint64_t jhi_slice = jlo + chunks_per_slice * kChebJ;
  const uint64_t jhi = jhi_slice < jend ? jhi_slice : jend;
  for (uint64_t j0 = jlo; j0 < jhi; j0 += kChebJ) {
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < kChebJ; t += kChebM) s_ij[t] = j0 + t < capacity ? ifact[j0 + t] : 0u;
    for (uint32_t t = threadIdx.x; t < kChebM + kChebJ; t += kChebM) {
      const uint64_t i = m0 + j0 + t;
      s_imj[t] = i < capacity ? ifact[i] : 0u;
    }
    for (uint32_t t = threadIdx.x; t < kChebM + 2 * kChebJ; t += kChebM) {
      const uint64_t k = m0 + 2 * j0 + t;
      s_ax[t] = k < count ? ax[k] : make_uint4(0u, 0u, 0u, 0u);
      s_ay[t] = k < count ? ay[k] : make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    if (m < capacity) {
#pragma unroll 4
      for (uint32_t t = 0; t < kChebJ; t++) {
        // term j = j0 + t: k = m + 2j sits at local index threadIdx.x + 2t, m + j at threadIdx.x + t
        const uint32_t w = m31_mul(s_ij[t], s_imj[threadIdx.x + t]);
        const uint4 vx = s_ax[threadIdx.x + 2 * t], vy = s_ay[threadIdx.x + 2 * t];
        sx = q_add(sx, q_mul_m31(qm31{vx.x, vx.y, vx.z, vx.w}, w));
        sy = q_add(sy, q_mul_m31(qm31{vy.x, vy.y, vy.z, vy.w}, w));
      }
    }
  }
  if (m >= capacity) return;
  const uint64_t o = (uint64_t)blockIdx.y * capacity + m;
  px[o] = make_uint4(sx.a, sx.b, sx.c, sx.d);
  py[o] = make_uint4(sy.a, sy.b, sy.c, sy.d);
}

// c_m = sum of the slices' partial sums, halved for m = 0.
__global__ void chebyshev_sum_kernel(const uint4* __restrict__ px, const uint4* __restrict__ py, uint32_t slices, uint4* __restrict__ cx,
                                     uint4* __restrict__ cy, uint64_t capacity) {
  const uint64_t m = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= capacity) return;
  qm31 sx = {0, 0, 0, 0}, sy = {0, 0, 0, 0};
  for (uint32_t y = 0; y < slices; y++) {
    const uint4 vx = px[(uint64_t)y * capacity + m], vy = py[(uint64_t)y * capacity + m];
    sx = q_add(sx, qm31{vx.x, vx.y, vx.z, vx.w});
    sy = q_add(sy, qm31{vy.x, vy.y, vy.z, vy.w});
  }
  if (m == 0) {
    sx = q_mul_m31(sx, kInv2);
    sy = q_mul_m31(sy, kInv2);
  }
  cx[m] = make_uint4(sx.a, sx.b, sx.c, sx.d);
  cy[m] = make_uint4(sy.a, sy.b, sy.c, sy.d);
}

__device__ __forceinline__ void line_pair(uint4& lo, uint4& hi) {
  const qm31 l = {lo.x, lo.y, lo.z, lo.w}, h = {hi.x, hi.y, hi.z, hi.w};
  const qm31 nl = q_sub(l, h), nh = q_add(h, h);
  lo = make_uint4(nl.a, nl.b, nl.c, nl.d);
  hi = make_uint4(nh.a, nh.b, nh.c, nh.d);
}

// One level of the Chebyshev -> line-basis recursion for blocks of size s > 1024:
// pair (i, s - i), 1 <= i < s/2, of every block.
__global__ void line_level_kernel(uint4* __restrict__ v, uint64_t n, uint64_t s) {
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t half = s >> 1;
  const uint64_t per = half - 1;  // pairs per block
  if (per == 0 || g >= (n / s) * per) return;
  const uint64_t b = g / per, i = g % per + 1;
  uint4 lo = v[b * s + i], hi = v[b * s + s - i];
  line_pair(lo, hi);
  v[b * s + i] = lo;
  v[b * s + s - i] = hi;
}

// The levels s <= 1024 of one 1024-value tile (or the whole vector if shorter) in
// shared memory, for both columns, then the interleaved output
// out[2i] = x line basis, out[2i+1] = y line basis.
static constexpr uint32_t kLineTile = 1024;  // 2 x 16 KiB of static shared memory

__global__ void __launch_bounds__(512) line_tile_kernel(const uint4* __restrict__ cx, const uint4* __restrict__ cy, uint64_t n, uint32_t top,
                                                         uint4* __restrict__ out) {
  __shared__ uint4 sx[kLineTile], sy[kLineTile];
  const uint32_t T = n < kLineTile ? (uint32_t)n : kLineTile;
  const uint64_t base = (uint64_t)blockIdx.x * T;
  for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
    sx[t] = cx[base + t];
    sy[t] = cy[base + t];
  }
  __syncthreads();
  for (uint32_t s = top; s >= 2; s >>= 1) {
    const uint32_t half = s >> 1, per = half - 1;
    for (uint32_t g = threadIdx.x; g < (T / s) * per; g += blockDim.x) {
      const uint32_t b = g / per, i = g % per + 1;
      line_pair(sx[b * s + i], sx[b * s + s - i]);
      line_pair(sy[b * s + i], sy[b * s + s - i]);
    }
    __syncthreads();
  }
  for (uint32_t t = threadIdx.x; t < T; t += blockDim.x) {
    out[2 * (base + t)] = sx[t];
    out[2 * (base + t) + 1] = sy[t];
  }
}

cudaError_t launch_witness_tables(uint64_t n, uint32_t* fact, uint32_t* seg, uint32_t* ifact, uint32_t* scale, cudaStream_t s) {
  const uint32_t nseg = (uint32_t)((n + 1023) / 1024);
  fact_segments_kernel<<<nseg, 1024, 0, s>>>(fact, seg, n);
  fact_seg_prefix_kernel<<<1, 32, 0, s>>>(seg, nseg);
  fact_finish_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(fact, seg, ifact, scale, n);
  return cudaGetLastError();
}

// Slices of the j range so that the Chebyshev launch has about two blocks per SM
// (at least one chunk of kChebJ terms per slice).
static uint32_t chebyshev_slices(uint64_t n, uint64_t count) {
  const uint64_t mblocks = (n + kChebM - 1) / kChebM;
  const uint64_t chunks = ((count + 1) / 2 + kChebJ - 1) / kChebJ;
  uint64_t y = (kWitnessBlockTarget + mblocks - 1) / mblocks;
  if (y > chunks) y = chunks;
  return (uint32_t)(y ? y : 1);
}

uint64_t witness_partial_values(uint64_t n) {
  // slices * n <= (kWitnessBlockTarget / mblocks + 1) * n <= kWitnessBlockTarget * kChebM + n
  return (uint64_t)kWitnessBlockTarget * kChebM + n;
}

// x, y: count_x / count_y monomial coefficients (QM31); capacity n = half the
// domain; out: 2n QM31.  ax, ay, cx, cy: n QM31 each of scratch; px, py:
// witness_partial_values(n) QM31 each.
cudaError_t launch_witness_transform(const uint4* x, uint64_t count_x, const uint4* y, uint64_t count_y, uint64_t n, const uint32_t* ifact,
                                     const uint32_t* scale, uint4* ax, uint4* ay, uint4* px, uint4* py, uint4* cx, uint4* cy, uint4* out,
                                     cudaStream_t s) {
  const uint64_t count = count_x > count_y ? count_x : count_y;
  witness_scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(x, count_x, scale, ax, n);
  witness_scale_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(y, count_y, scale, ay, n);
  const uint32_t slices = chebyshev_slices(n, count);
  const uint64_t chunks = ((count + 1) / 2 + kChebJ - 1) / kChebJ;
  const uint64_t per_slice = (chunks + slices - 1) / slices;
  chebyshev_kernel<<<dim3((unsigned)((n + kChebM - 1) / kChebM), slices), kChebM, 0, s>>>(ax, ay, count, ifact, px, py, n, per_slice ? per_slice : 1);
  chebyshev_sum_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(px, py, slices, cx, cy, n);
  for (uint64_t sz = n; sz > kLineTile; sz >>= 1) {
    const uint64_t pairs = (n / sz) * ((sz >> 1) - 1);
    line_level_kernel<<<(unsigned)((pairs + 255) / 256), 256, 0, s>>>(cx, n, sz);
    line_level_kernel<<<(unsigned)((pairs + 255) / 256), 256, 0, s>>>(cy, n, sz);
  }
  const uint32_t T = n < kLineTile ? (uint32_t)n : kLineTile;
  line_tile_kernel<<<(unsigned)(n / T), 512, 0, s>>>(cx, cy, n, T, out);
  return cudaGetLastError();
}

}  // namespace azk
