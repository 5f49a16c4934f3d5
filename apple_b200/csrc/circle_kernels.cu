// Circle domain tables, Circle FFT codeword, QM31 FRI folds and the Circle
// PCS/FRI transcript + proof emission kernels.
//
// References: domain and twiddles CircleDomain.swift:187-511 and
// CircleCodeword.swift:129-171 (Metal: HashMerkleKernels.metal:1720-1879); FFT
// CircleCodeword.swift:72-98 (Metal :1881-1943); fold QM31FRIFold.swift:11-44
// (Metal :1987-2032); transcript and proof layout CircleProofFormat.swift:475-983.
#include "azk_field.cuh"
#include "azk_internal.h"

namespace azk {

// ---------------------------------------------------------------------------
// Domain tables.  tw[off(s) + h] = stage-s FFT twiddle of block h (and tw[N + g]
// = 2 tw[g], the doubled copy the register-blocked FFT multiplies by), with
// off(0) = 0 and off(s) = N - (N >> s): the y coordinate of the point at storage
// index h << 1 for stage 0, else its x coordinate doubled s - 1 times.  The FRI
// inverse-domain layer k is the elementwise inverse of stage k (inv(y) for the
// circle-to-line fold, inv(x) of the left line point afterwards).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t tw_offset(uint32_t logn, uint32_t s) {
  uint64_t n = 1ull << logn;
  return s == 0 ? 0 : n - (n >> s);
}

__global__ void domain_tables_kernel(uint32_t logn, uint32_t* __restrict__ tw, uint32_t* __restrict__ inv) {
  uint64_t n = 1ull << logn;
  uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n - 1) return;
  uint32_t s = 0;
  while (g >= tw_offset(logn, s + 1)) s++;
  uint64_t h = g - tw_offset(logn, s);
  uint32_t nat = bit_reverse((uint32_t)(h << (s + 1)), logn);
  cpoint p = cp_from_index(circle_point_index(logn, nat));
  uint32_t v;
  if (s == 0) {
    v = p.y;
  } else {
    v = p.x;
    for (uint32_t k = 1; k < s; k++) v = double_x(v);
  }
  tw[g] = v;
  tw[n + g] = v << 1;  // doubled copy for the register-blocked FFT's multiply
  if (inv) inv[g] = m31_inv(v);
}

cudaError_t launch_domain_tables(uint32_t logn, uint32_t* d_tw, uint32_t* d_inv, cudaStream_t s) {
  uint64_t n = 1ull << logn;
  if (n < 2) return cudaSuccess;
  domain_tables_kernel<<<(unsigned)((n - 1 + 255) / 256), 256, 0, s>>>(logn, d_tw, d_inv);
  return cudaGetLastError();
}

__global__ void domain_points_kernel(uint32_t logn, uint32_t* __restrict__ xy) {
  uint64_t n = 1ull << logn;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cpoint p = cp_from_index(circle_point_index(logn, bit_reverse((uint32_t)i, logn)));
  xy[2 * i] = p.x;
  xy[2 * i + 1] = p.y;
}

cudaError_t launch_domain_points(uint32_t logn, uint32_t* d_xy, cudaStream_t s) {
  uint64_t n = 1ull << logn;
  domain_points_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(logn, d_xy);
  return cudaGetLastError();
}

// M31 values as QM31 values (a, 0, 0, 0): the inverse-domain layers in the
// 16-byte layout the QM31 fold plans take.
__global__ void widen_m31_kernel(const uint32_t* __restrict__ in, uint4* __restrict__ out, uint64_t n) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = make_uint4(__ldg(in + i), 0u, 0u, 0u);
}

cudaError_t launch_widen_m31(const uint32_t* d_in, uint4* d_out, uint64_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  uint64_t blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  widen_m31_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_in, d_out, n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Circle FFT.  Stages run logn-1 ... 0; stage s pairs (i, i + 2^s) inside blocks
// of 2^(s+1) with the block's twiddle t: (l + r t, l - r t).  A pass runs a range
// of m consecutive stages on shared-memory tiles of 2^m "rows" (the stage bits)
// by 2^c "columns" (the lowest index bits, for 64-byte coalesced rows).  The last
// pass (stages min(logn,12)-1 ... 0) uses contiguous 4096-element tiles; the
// stages above 12 run first in chunks of at most 10.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t fft_global_index(const FftPassGeom& g, uint64_t tile, uint32_t L) {
  uint32_t row = L >> g.c, col = L & ((1u << g.c) - 1);
  uint32_t midbits = g.s_lo > g.c ? g.s_lo - g.c : 0;
  uint64_t mid = tile & ((1ull << midbits) - 1);
  uint64_t hi = tile >> midbits;
  return (hi << (g.s_lo + g.m)) | ((uint64_t)row << g.s_lo) | (mid << g.c) | col;
}

// Stage j of a pass (global stage s_lo + j) pairs local indices that differ in bit
// j + c, and its twiddle is tw[off(s) + (gi >> (s + 1))] = tw[off(s) + (hi <<
// (m-1-j)) + (row >> (j + 1))]: 2^(m-1-j) consecutive table entries per tile,
// staged in shared memory at stw + 2^m - 2^(m-j).  Shared arrays are padded by
// one word per 32 so the strided butterfly groups spread over the banks.
__device__ __forceinline__ uint32_t fft_stw_offset(uint32_t m, uint32_t j) { return (1u << m) - (1u << (m - j)); }
__device__ __forceinline__ uint32_t fpad(uint32_t L) { return L + (L >> 5); }

struct FftTile {
  FftPassGeom g;
  uint32_t T;
  uint64_t count;
  bool first, last;
  bool top_zero;  // first pass over a nonzero prefix of at most N/4 (see fft_m31_tile_stages)
};

__device__ __forceinline__ FftTile fft_tile(const FftJob& job) {
  FftTile t;
  t.g = fft_pass_geom(job.logn, job.pass);
  t.T = 1u << (t.g.m + t.g.c);
  const uint64_t N = 1ull << job.logn;
  t.count = (job.info != nullptr && job.info->count != 0) ? job.info->count : N;
  t.first = job.pass == 0;
  t.last = job.pass == fft_high_chunks(job.logn);
  t.top_zero = t.first && job.logn >= 2 && t.count <= (N >> 2);
  return t;
}

template <int THREADS>
__device__ __forceinline__ void fft_stage_twiddles(const FftJob& job, const FftTile& ft, uint64_t tile, uint32_t* stw) {
  const FftPassGeom& g = ft.g;
  const uint32_t midbits = g.s_lo > g.c ? g.s_lo - g.c : 0;
  const uint64_t hi = tile >> midbits;
  for (uint32_t j = 0; j < g.m; j++) {
    const uint32_t cnt = 1u << (g.m - 1 - j);
    const uint32_t* src = job.tw + tw_offset(job.logn, g.s_lo + j) + (hi << (g.m - 1 - j));
    uint32_t* dst = stw + fft_stw_offset(g.m, j);
    for (uint32_t r = threadIdx.x; r < cnt; r += THREADS) dst[r] = __ldg(src + r);
  }
}

__device__ __forceinline__ void bfly_m31(uint32_t& l, uint32_t& r, uint32_t t) {
  uint32_t rt = m31_mul(r, t);
  uint32_t a = m31_add(l, rt);
  r = m31_sub(l, rt);
  l = a;
}

__device__ __forceinline__ void bfly_q(qm31& l, qm31& r, uint32_t t) {
  qm31 rt = q_mul_m31(r, t);
  qm31 a = q_add(l, rt);
  r = q_sub(l, rt);
  l = a;
}

// QM31 tiles: the four limbs as four padded u32 arrays; two stages per
// shared-memory round trip (radix 4 in registers), then one more if m is odd.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) fft_pass_q_kernel(const FftJob* __restrict__ jobs, const uint2* __restrict__ work) {
  extern __shared__ uint32_t fsm[];
  const uint2 w = work[blockIdx.x];
  const FftJob& job = jobs[w.x];
  const FftTile ft = fft_tile(job);
  const FftPassGeom& g = ft.g;
  const uint32_t T = ft.T, TP = T + (T >> 5);
  uint32_t* sa = fsm;
  uint32_t* sb = sa + TP;
  uint32_t* sc = sb + TP;
  uint32_t* sd = sc + TP;
  uint32_t* stw = sd + TP;
  fft_stage_twiddles<THREADS>(job, ft, w.y, stw);
  // tile index L = threadIdx.x + k * THREADS: the global index advances by a constant
  const uint64_t gstep = (uint64_t)(THREADS >> g.c) << g.s_lo;
  const uint64_t gi0 = fft_global_index(g, w.y, threadIdx.x);
  {
    uint64_t gi = gi0;
    for (uint32_t L = threadIdx.x; L < T; L += THREADS, gi += gstep) {
      uint4 v;
      if (ft.first)
        v = gi < ft.count ? __ldg(job.in + gi) : make_uint4(0u, 0u, 0u, 0u);
      else
        v = job.out[gi];
      const uint32_t a = fpad(L);
      sa[a] = v.x;
      sb[a] = v.y;
      sc[a] = v.z;
      sd[a] = v.w;
    }
  }
  __syncthreads();
  int j = (int)g.m - 1;
  for (; j >= 1; j -= 2) {
    const uint32_t p = (uint32_t)j + g.c;  // stage j pairs bit p, stage j-1 pairs bit p-1
    const uint32_t* tw_j = stw + fft_stw_offset(g.m, (uint32_t)j);
    const uint32_t* tw_j1 = stw + fft_stw_offset(g.m, (uint32_t)j - 1);
    const uint32_t lowmask = (1u << (p - 1)) - 1;
    const uint32_t o1 = fpad(1u << (p - 1)), o2 = fpad(1u << p), o3 = fpad(3u << (p - 1));
    for (uint32_t k = threadIdx.x; k < T / 4; k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << 2) | (k & lowmask);
      const uint32_t row = e0 >> g.c;
      const uint32_t t1 = tw_j[row >> (j + 1)];
      const uint32_t t2a = tw_j1[row >> j], t2b = tw_j1[(row >> j) | 1u];
      const uint32_t a0 = fpad(e0), a1 = a0 + o1, a2 = a0 + o2, a3 = a0 + o3;
      qm31 v0 = {sa[a0], sb[a0], sc[a0], sd[a0]}, v1 = {sa[a1], sb[a1], sc[a1], sd[a1]};
      qm31 v2 = {sa[a2], sb[a2], sc[a2], sd[a2]}, v3 = {sa[a3], sb[a3], sc[a3], sd[a3]};
      bfly_q(v0, v2, t1);
      bfly_q(v1, v3, t1);
      bfly_q(v0, v1, t2a);
      bfly_q(v2, v3, t2b);
      sa[a0] = v0.a, sb[a0] = v0.b, sc[a0] = v0.c, sd[a0] = v0.d;
      sa[a1] = v1.a, sb[a1] = v1.b, sc[a1] = v1.c, sd[a1] = v1.d;
      sa[a2] = v2.a, sb[a2] = v2.b, sc[a2] = v2.c, sd[a2] = v2.d;
      sa[a3] = v3.a, sb[a3] = v3.b, sc[a3] = v3.c, sd[a3] = v3.d;
    }
    __syncthreads();
  }
  if (j == 0) {
    const uint32_t p = g.c;
    for (uint32_t k = threadIdx.x; k < T / 2; k += THREADS) {
      const uint32_t L = ((k >> p) << (p + 1)) | (k & ((1u << p) - 1));
      const uint32_t t = stw[(L >> g.c) >> 1];
      const uint32_t aL = fpad(L), aR = fpad(L | (1u << p));
      qm31 l = {sa[aL], sb[aL], sc[aL], sd[aL]}, r = {sa[aR], sb[aR], sc[aR], sd[aR]};
      bfly_q(l, r, t);
      sa[aL] = l.a, sb[aL] = l.b, sc[aL] = l.c, sd[aL] = l.d;
      sa[aR] = r.a, sb[aR] = r.b, sc[aR] = r.c, sd[aR] = r.d;
    }
    __syncthreads();
  }
  {
    uint64_t gi = gi0;
    for (uint32_t L = threadIdx.x; L < T; L += THREADS, gi += gstep) {
      const uint32_t a = fpad(L);
      job.out[gi] = make_uint4(sa[a], sb[a], sc[a], sd[a]);
    }
  }
}

// One-limb tiles for inputs that are lifted M31 polynomials (b = c = d = 0 in
// every coefficient, so in every intermediate value): the first pass reads the
// a limbs of the nonzero prefix, passes exchange one word per element through
// `narrow`, and the last pass writes the QM31 codeword (a, 0, 0, 0).  Three stages
// per shared-memory round trip (radix 8 in registers).
// The stages of one one-limb tile (2^m rows x 2^c columns, values in `sv` with one
// pad word per 32, stage twiddles in `stw`), three per shared-memory round trip.
// Starts after and ends with a __syncthreads.  `top_zero`: the tile holds the
// transform's two top stages and every value whose row has either of the two top
// bits set is zero (a first pass whose nonzero prefix is at most N/4, as at blowup
// 4).  Those two stages then only copy (l + 0 t, l - 0 t), so the first round trip
// reads 2 of its 8 values and runs 4 of its 12 butterflies.
template <int THREADS>
__device__ __forceinline__ void fft_m31_tile_stages(uint32_t* sv, const uint32_t* stw, const FftPassGeom& g, uint32_t T, bool top_zero) {
  int j = (int)g.m - 1;
  if (top_zero && g.m % 3 == 1 && j >= 3) {
    // m = 4, 7, 10: the two copying stages and the next two (radix 4 on the 4 live
    // values of a 16-value group, once per copy) in one round trip, so the rest is
    // whole radix-8 trips instead of ending on a one-stage trip
    const uint32_t p = (uint32_t)j + g.c;
    const uint32_t* tw2 = stw + fft_stw_offset(g.m, (uint32_t)j - 2);
    const uint32_t* tw3 = stw + fft_stw_offset(g.m, (uint32_t)j - 3);
    const uint32_t lowmask = (1u << (p - 3)) - 1;
    uint32_t ob[16];
#pragma unroll
    for (uint32_t b = 0; b < 16; b++)
      ob[b] = fpad(((b >> 3) << p) | (((b >> 2) & 1u) << (p - 1)) | (((b >> 1) & 1u) << (p - 2)) | ((b & 1u) << (p - 3)));
    for (uint32_t k = threadIdx.x; k < T / 16; k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << 4) | (k & lowmask);
      const uint32_t row = e0 >> g.c;
      const uint32_t a0 = fpad(e0);
      const uint32_t x0 = sv[a0], x1 = sv[a0 + ob[1]], x2 = sv[a0 + ob[2]], x3 = sv[a0 + ob[3]];
      const uint32_t r2 = row >> (j - 1), r3 = row >> (j - 2);
#pragma unroll
      for (uint32_t q = 0; q < 4; q++) {
        // copy q of the live values (its two top row bits = q)
        const uint32_t t2 = tw2[r2 | q];
        uint32_t y0 = x0, y1 = x1, y2 = x2, y3 = x3;
        bfly_m31(y0, y2, t2);
        bfly_m31(y1, y3, t2);
        bfly_m31(y0, y1, tw3[r3 | (q << 1)]);
        bfly_m31(y2, y3, tw3[r3 | (q << 1) | 1u]);
        sv[a0 + ob[4 * q]] = y0;
        sv[a0 + ob[4 * q + 1]] = y1;
        sv[a0 + ob[4 * q + 2]] = y2;
        sv[a0 + ob[4 * q + 3]] = y3;
      }
    }
    __syncthreads();
    j -= 4;
  } else if (top_zero && j >= 2) {
    const uint32_t p = (uint32_t)j + g.c;
    const uint32_t* tw2 = stw + fft_stw_offset(g.m, (uint32_t)j - 2);
    const uint32_t lowmask = (1u << (p - 2)) - 1;
    uint32_t ob[8];
#pragma unroll
    for (uint32_t b = 0; b < 8; b++) ob[b] = fpad(((b >> 2) << p) | (((b >> 1) & 1u) << (p - 1)) | ((b & 1u) << (p - 2)));
    for (uint32_t k = threadIdx.x; k < T / 8; k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << 3) | (k & lowmask);
      const uint32_t row = e0 >> g.c;
      const uint32_t a0 = fpad(e0);
      const uint32_t x0 = sv[a0], x1 = sv[a0 + ob[1]];
      const uint32_t r2 = row >> (j - 1);
#pragma unroll
      for (uint32_t q = 0; q < 4; q++) {
        // after the two copying stages the pair (2q, 2q + 1) holds (x0, x1)
        uint32_t l = x0, r = x1;
        bfly_m31(l, r, tw2[r2 | q]);
        sv[a0 + ob[2 * q]] = l;
        sv[a0 + ob[2 * q + 1]] = r;
      }
    }
    __syncthreads();
    j -= 3;
  } else if (top_zero && j >= 0) {
    // one or two stages, both copying: every value of a group takes its live one
    const uint32_t p = (uint32_t)j + g.c;
    const uint32_t span = 1u << (p - (uint32_t)j);  // the live row's stride: the group is {e0 + span * b}
    const uint32_t bits = (uint32_t)j + 1;
    const uint32_t lowmask = span - 1;
    for (uint32_t k = threadIdx.x; k < (T >> bits); k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << bits) | (k & lowmask);
      const uint32_t x = sv[fpad(e0)];
      for (uint32_t b = 1; b < (1u << bits); b++) sv[fpad(e0 + span * b)] = x;
    }
    __syncthreads();
    return;
  }
  for (; j >= 2; j -= 3) {
    const uint32_t p = (uint32_t)j + g.c;  // stages j, j-1, j-2 pair bits p, p-1, p-2
    const uint32_t* tw0 = stw + fft_stw_offset(g.m, (uint32_t)j);
    const uint32_t* tw1 = stw + fft_stw_offset(g.m, (uint32_t)j - 1);
    const uint32_t* tw2 = stw + fft_stw_offset(g.m, (uint32_t)j - 2);
    const uint32_t lowmask = (1u << (p - 2)) - 1;
    // the group's 8 indices are e0 with bits p, p-1, p-2 set per b; e0 has those
    // bits clear, so fpad(e0 | o) = fpad(e0) + fpad(o)
    uint32_t ob[8];
#pragma unroll
    for (uint32_t b = 0; b < 8; b++) ob[b] = fpad(((b >> 2) << p) | (((b >> 1) & 1u) << (p - 1)) | ((b & 1u) << (p - 2)));
    for (uint32_t k = threadIdx.x; k < T / 8; k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << 3) | (k & lowmask);
      const uint32_t row = e0 >> g.c;
      const uint32_t a0 = fpad(e0);
      uint32_t a[8], v[8];
#pragma unroll
      for (uint32_t b = 0; b < 8; b++) {
        a[b] = a0 + ob[b];
        v[b] = sv[a[b]];
      }
      const uint32_t t0 = tw0[row >> (j + 1)];
      const uint32_t r1 = row >> j, r2 = row >> (j - 1);
      const uint32_t t1a = tw1[r1], t1b = tw1[r1 | 1u];
      const uint32_t t2a = tw2[r2], t2b = tw2[r2 | 1u], t2c = tw2[r2 | 2u], t2d = tw2[r2 | 3u];
      bfly_m31(v[0], v[4], t0);
      bfly_m31(v[1], v[5], t0);
      bfly_m31(v[2], v[6], t0);
      bfly_m31(v[3], v[7], t0);
      bfly_m31(v[0], v[2], t1a);
      bfly_m31(v[1], v[3], t1a);
      bfly_m31(v[4], v[6], t1b);
      bfly_m31(v[5], v[7], t1b);
      bfly_m31(v[0], v[1], t2a);
      bfly_m31(v[2], v[3], t2b);
      bfly_m31(v[4], v[5], t2c);
      bfly_m31(v[6], v[7], t2d);
#pragma unroll
      for (uint32_t b = 0; b < 8; b++) sv[a[b]] = v[b];
    }
    __syncthreads();
  }
  if (j == 1) {
    const uint32_t p = 1u + g.c;
    const uint32_t* tw0 = stw + fft_stw_offset(g.m, 1);
    const uint32_t lowmask = (1u << (p - 1)) - 1;
    for (uint32_t k = threadIdx.x; k < T / 4; k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << 2) | (k & lowmask);
      const uint32_t row = e0 >> g.c;
      const uint32_t t1 = tw0[row >> 2];
      const uint32_t t2a = stw[row >> 1], t2b = stw[(row >> 1) | 1u];
      const uint32_t a0 = fpad(e0), a1 = fpad(e0 | (1u << (p - 1))), a2 = fpad(e0 | (1u << p)), a3 = fpad(e0 | (3u << (p - 1)));
      uint32_t v0 = sv[a0], v1 = sv[a1], v2 = sv[a2], v3 = sv[a3];
      bfly_m31(v0, v2, t1);
      bfly_m31(v1, v3, t1);
      bfly_m31(v0, v1, t2a);
      bfly_m31(v2, v3, t2b);
      sv[a0] = v0;
      sv[a1] = v1;
      sv[a2] = v2;
      sv[a3] = v3;
    }
    __syncthreads();
  } else if (j == 0) {
    const uint32_t p = g.c;
    for (uint32_t k = threadIdx.x; k < T / 2; k += THREADS) {
      const uint32_t L = ((k >> p) << (p + 1)) | (k & ((1u << p) - 1));
      const uint32_t t = stw[(L >> g.c) >> 1];
      const uint32_t aL = fpad(L), aR = fpad(L | (1u << p));
      uint32_t l = sv[aL], r = sv[aR];
      bfly_m31(l, r, t);
      sv[aL] = l;
      sv[aR] = r;
    }
    __syncthreads();
  }
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) fft_pass_m31_kernel(const FftJob* __restrict__ jobs, const uint2* __restrict__ work) {
  extern __shared__ uint32_t nsm[];
  const uint2 w = work[blockIdx.x];
  const FftJob& job = jobs[w.x];
  const FftTile ft = fft_tile(job);
  const FftPassGeom& g = ft.g;
  const uint32_t T = ft.T;
  uint32_t* sv = nsm;
  uint32_t* stw = sv + T + (T >> 5);
  fft_stage_twiddles<THREADS>(job, ft, w.y, stw);
  const uint32_t* in_a = reinterpret_cast<const uint32_t*>(job.in);
  // tile index L = threadIdx.x + k * THREADS: the rows advance by THREADS >> c, so
  // the global index advances by a constant
  const uint64_t gstep = (uint64_t)(THREADS >> g.c) << g.s_lo;
  const uint64_t gi0 = fft_global_index(g, w.y, threadIdx.x);
  {
    uint64_t gi = gi0;
    for (uint32_t L = threadIdx.x; L < T; L += THREADS, gi += gstep) {
      uint32_t v;
      if (ft.first)
        v = gi < ft.count ? __ldg(in_a + 4 * gi) : 0u;
      else
        v = job.narrow[gi];
      sv[fpad(L)] = v;
    }
  }
  __syncthreads();
  fft_m31_tile_stages<THREADS>(sv, stw, g, T, ft.top_zero);
  {
    uint64_t gi = gi0;
    for (uint32_t L = threadIdx.x; L < T; L += THREADS, gi += gstep) {
      const uint32_t v = sv[fpad(L)];
      if (ft.last)
        job.out[gi] = make_uint4(v, 0u, 0u, 0u);
      else
        job.narrow[gi] = v;
    }
  }
}

// tiles of at most 4096 values (+ one pad word per 32) and 4095 staged twiddles
static constexpr uint32_t kFftTileMax = 1u << kFftLowBits;
static constexpr uint32_t kFftTilePadded = kFftTileMax + (kFftTileMax >> 5);
static constexpr size_t kFftSmemQ = (size_t)4 * (4 * kFftTilePadded + kFftTileMax);
static constexpr size_t kFftSmemM31 = (size_t)4 * (kFftTilePadded + kFftTileMax);
static constexpr int kFftThreadsQ = 512;
static constexpr int kFftThreadsM31 = 256;

cudaError_t prepare_fft_kernels() {
  cudaError_t e = cudaFuncSetAttribute(fft_pass_q_kernel<kFftThreadsQ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFftSmemQ);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fft_pass_m31_kernel<kFftThreadsM31>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFftSmemM31);
  if (e != cudaSuccess) return e;
  return prepare_fft_m31_kernels();
}

cudaError_t launch_fft_pass(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t kind, uint32_t* d_status, cudaStream_t s) {
  if (nwork == 0) return cudaSuccess;
  switch (kind) {
    case kFftQM31:
      fft_pass_q_kernel<kFftThreadsQ><<<nwork, kFftThreadsQ, kFftSmemQ, s>>>(d_jobs, d_work);
      break;
    case kFftM31Small:
      fft_pass_m31_kernel<kFftThreadsM31><<<nwork, kFftThreadsM31, kFftSmemM31, s>>>(d_jobs, d_work);
      break;
    case kFftM31Tile:
      return launch_fft_m31_tiles(d_jobs, d_work, nwork, s);
    case kFftM31Low:
      return launch_fft_m31_low(d_jobs, d_work, nwork, d_status, s);
    case kFftQ4Tile:
      return launch_fft_q_tiles(d_jobs, d_work, nwork, s);
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Folds (one thread per output pair)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) fold_kernel(const FoldJob* __restrict__ jobs, const uint2* __restrict__ work) {
  const uint2 w = work[blockIdx.x];
  const FoldJob& job = jobs[w.x];
  __shared__ uint32_t s_ch[4];
  if (threadIdx.x < 4) s_ch[threadIdx.x] = __ldcg(job.ch + threadIdx.x);
  __syncthreads();
  const qm31 ch = {s_ch[0], s_ch[1], s_ch[2], s_ch[3]};
  uint64_t base = (uint64_t)w.y * kFoldChunk;
  for (uint32_t k = threadIdx.x; k < kFoldChunk; k += blockDim.x) {
    uint64_t i = base + k;
    if (i >= job.n_out) break;
    uint4 p = __ldg(job.prev + 2 * i), q = __ldg(job.prev + 2 * i + 1);
    qm31 r = fri_fold_pair(qm31{p.x, p.y, p.z, p.w}, qm31{q.x, q.y, q.z, q.w}, __ldg(job.inv + i), ch);
    job.out[i] = make_uint4(r.a, r.b, r.c, r.d);
  }
}

cudaError_t launch_fold_jobs(const FoldJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s) {
  if (nwork == 0) return cudaSuccess;
  fold_kernel<<<nwork, 256, 0, s>>>(d_jobs, d_work);
  return cudaGetLastError();
}

// Fold with a QM31 inverse-domain layer given as full QM31 values (the QM31 fold
// plan API takes arbitrary QM31 inverse points, QM31FRIFold.swift:960-1338).
// The challenge is read once per block into shared memory; a grid-stride loop
// with two outputs per step keeps two sets of loads in flight per thread.
__global__ void __launch_bounds__(256) fold_qm31_inv_kernel(const uint4* __restrict__ prev, const uint4* __restrict__ inv,
                                                            const uint32_t* __restrict__ chp, uint4* __restrict__ out, uint64_t n_out) {
  __shared__ uint32_t s_ch[4];
  if (threadIdx.x < 4) s_ch[threadIdx.x] = __ldcg(chp + threadIdx.x);
  __syncthreads();
  const qm31 ch = {s_ch[0], s_ch[1], s_ch[2], s_ch[3]};
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_out; i += 2 * stride) {
    const uint64_t i2 = i + stride;
    const bool two = i2 < n_out;
    const uint4 p = __ldg(prev + 2 * i), q = __ldg(prev + 2 * i + 1), t = __ldg(inv + i);
    uint4 p2 = p, q2 = q, t2 = t;
    if (two) {
      p2 = __ldg(prev + 2 * i2);
      q2 = __ldg(prev + 2 * i2 + 1);
      t2 = __ldg(inv + i2);
    }
    {
      qm31 pos = {p.x, p.y, p.z, p.w}, neg = {q.x, q.y, q.z, q.w};
      qm31 odd = q_mul(q_sub(pos, neg), qm31{t.x, t.y, t.z, t.w});
      qm31 r = q_half(q_add(q_add(pos, neg), q_mul(ch, odd)));
      out[i] = make_uint4(r.a, r.b, r.c, r.d);
    }
    if (two) {
      qm31 pos = {p2.x, p2.y, p2.z, p2.w}, neg = {q2.x, q2.y, q2.z, q2.w};
      qm31 odd = q_mul(q_sub(pos, neg), qm31{t2.x, t2.y, t2.z, t2.w});
      qm31 r = q_half(q_add(q_add(pos, neg), q_mul(ch, odd)));
      out[i2] = make_uint4(r.a, r.b, r.c, r.d);
    }
  }
}

cudaError_t launch_fold_qm31_inv(const uint4* prev, const uint4* inv, const uint32_t* ch, uint4* out, uint64_t n_out, cudaStream_t s) {
  if (n_out == 0) return cudaSuccess;
  uint64_t blocks = (n_out + 511) / 512;
  if (blocks > 148 * 16) blocks = 148 * 16;
  fold_qm31_inv_kernel<<<(unsigned)blocks, 256, 0, s>>>(prev, inv, ch, out, n_out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Circle FRI PCS V1 transcript (CircleProofFormat.swift:684-983)
// ---------------------------------------------------------------------------
__device__ void absorb_domain_codec(Transcript& t, uint32_t logn) {
  // CircleDomainDescriptorCodecV1.encode (CircleProofFormat.swift:75-93)
  FrameBuf f;
  f.n = 0;
  const uint8_t magic[8] = {0x41, 0x5a, 0x4b, 0x43, 0x44, 0x56, 0x31, 0x00};
  for (int i = 0; i < 8; i++) fb_u8(f, magic[i]);
  fb_u32(f, 1);
  fb_u32(f, kP);
  fb_u32(f, 31);
  fb_u32(f, 2);
  fb_u32(f, 1268011823u);
  fb_u32(f, logn);
  fb_u32(f, (uint32_t)((1ull << (31 - (logn + 1))) & 0x7FFFFFFFu));
  fb_u32(f, logn - 1);
  fb_u32(f, 1);
  tr_absorb(t, f.b, f.n);
}

__global__ void pcs_prefix_kernel(PcsInstance* __restrict__ inst, uint32_t ninst) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ninst) return;
  PcsInstance& I = inst[i];
  Transcript t;
  tr_reset(t);
  FrameBuf f;
  circle_frame(f, 0);  // header
  fb_u32(f, 1);
  fb_u32(f, 1);
  fb_u32(f, kP);
  fb_u32(f, 2);
  fb_u32(f, 1268011823u);
  tr_absorb(t, f.b, f.n);
  absorb_domain_codec(t, I.logn);
  circle_frame(f, 1);  // security
  fb_u32(f, I.log_blowup);
  fb_u32(f, I.queries);
  fb_u32(f, 1);
  fb_u32(f, I.grinding_bits);
  fb_u32(f, I.log_blowup * I.queries + I.grinding_bits);
  tr_absorb(t, f.b, f.n);
  circle_frame(f, 2);  // public input
  fb_u32(f, 32);
  tr_absorb(t, f.b, f.n);
  uint64_t pub[4] = {I.pub[0], I.pub[1], I.pub[2], I.pub[3]};
  tr_absorb_digest(t, pub);
  *I.transcript = t;
}

cudaError_t launch_pcs_prefix(PcsInstance* d_inst, uint32_t ninst, cudaStream_t s) {
  if (!ninst) return cudaSuccess;
  pcs_prefix_kernel<<<(ninst + 63) / 64, 64, 0, s>>>(d_inst, ninst);
  return cudaGetLastError();
}

// Final-layer binding: frame (count, bytes) then the packed final layer.
__global__ void pcs_finalize_kernel(PcsInstance* __restrict__ inst, const uint32_t* __restrict__ ids, uint32_t nids) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nids) return;
  PcsInstance& I = inst[ids[j]];
  Transcript t = *I.transcript;
  uint64_t cnt = 1ull << (I.logn - I.rounds);
  FrameBuf f;
  circle_frame(f, 5);
  fb_u64(f, cnt);
  fb_u64(f, cnt * 16);
  tr_absorb(t, f.b, f.n);
  const uint8_t* fl = reinterpret_cast<const uint8_t*>(I.layers + layer_offset(I.logn, I.rounds));
  tr_absorb(t, fl, (uint32_t)(cnt * 16));
  *I.transcript = t;
}

cudaError_t launch_pcs_finalize(PcsInstance* d_inst, const uint32_t* d_ids, uint32_t nids, cudaStream_t s) {
  if (!nids) return cudaSuccess;
  pcs_finalize_kernel<<<(nids + 63) / 64, 64, 0, s>>>(d_inst, d_ids, nids);
  return cudaGetLastError();
}

__device__ __forceinline__ void absorb_grinding(Transcript& t, uint32_t bits, uint64_t nonce) {
  FrameBuf f;
  circle_frame(f, 7);
  fb_u32(f, bits);
  fb_u32(f, 8);
  tr_absorb(t, f.b, f.n);
  f.n = 0;
  fb_u64(f, nonce);
  tr_absorb(t, f.b, f.n);
}
// digestMeetsTarget (CircleProofFormat.swift:662-681): leading `bits` bits zero.
__device__ __forceinline__ bool grinding_ok(const Transcript& t, uint32_t bits) {
  uint8_t d[32];
  tr_squeeze_bytes(t, 32, d);
  int rem = (int)bits, i = 0;
  while (rem >= 8) {
    if (d[i]) return false;
    i++;
    rem -= 8;
  }
  if (rem == 0) return true;
  uint8_t mask = (uint8_t)(0xFF << (8 - rem));
  return (d[i] & mask) == 0;
}

__global__ void pcs_grind_kernel(const PcsInstance* __restrict__ inst, uint32_t id, uint64_t start, uint64_t count, unsigned long long* found) {
  uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const PcsInstance& I = inst[id];
  Transcript t = *I.transcript;
  uint64_t nonce = start + k;
  absorb_grinding(t, I.grinding_bits, nonce);
  if (grinding_ok(t, I.grinding_bits)) atomicMin(found, (unsigned long long)nonce);
}

cudaError_t launch_pcs_grind(PcsInstance* d_inst, uint32_t id, uint64_t start, uint64_t count, unsigned long long* d_found, cudaStream_t s) {
  pcs_grind_kernel<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(d_inst, id, start, count, d_found);
  return cudaGetLastError();
}

// Optional grinding absorb, then the query frame and q pair indices mod N/2.
__global__ void pcs_queries_kernel(PcsInstance* __restrict__ inst, const uint32_t* __restrict__ ids, uint32_t nids) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nids) return;
  PcsInstance& I = inst[ids[j]];
  Transcript t = *I.transcript;
  if (I.has_nonce) absorb_grinding(t, I.grinding_bits, I.nonce);
  FrameBuf f;
  circle_frame(f, 6);
  fb_u32(f, I.queries);
  fb_u64(f, 1ull << (I.logn - 1));
  tr_absorb(t, f.b, f.n);
  tr_squeeze_u32(t, I.queries, 1u << (I.logn - 1), I.query_pairs);
  *I.transcript = t;
}

cudaError_t launch_pcs_queries(PcsInstance* d_inst, const uint32_t* d_ids, uint32_t nids, cudaStream_t s) {
  if (!nids) return cudaSuccess;
  pcs_queries_kernel<<<(nids + 63) / 64, 64, 0, s>>>(d_inst, d_ids, nids);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Proof bytes (CirclePCSFRIProofCodecV1.encode, CircleProofFormat.swift:478-593).
// Every field starts at a 4-byte multiple, so the proof is written with u32
// stores: block (instance, q) writes query q; block (instance, queries) the
// header, the claimed openings and the nonce.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pw32(uint8_t* b, uint64_t off, uint32_t v) { *reinterpret_cast<uint32_t*>(b + off) = v; }
__device__ __forceinline__ void pw64(uint8_t* b, uint64_t off, uint64_t v) {
  pw32(b, off, (uint32_t)v);
  pw32(b, off + 4, (uint32_t)(v >> 32));
}
__device__ __forceinline__ void pwdig(uint8_t* b, uint64_t off, const uint64_t (&d)[4]) {
  for (int k = 0; k < 4; k++) pw64(b, off + 8 * k, d[k]);
}

// Sibling digest of leaf `idx` at `level` in tree k of an instance.
__device__ void pcs_sibling(const PcsInstance& I, uint32_t k, uint64_t idx, uint32_t level, uint64_t (&d)[4]) {
  uint32_t depth = I.logn - k;
  uint64_t node = (idx >> level) ^ 1ull;
  if (level == 0) {
    uint4 v = I.layers[layer_offset(I.logn, k) + node];
    sha3_16((uint64_t)v.x | ((uint64_t)v.y << 32), (uint64_t)v.z | ((uint64_t)v.w << 32), d);
  } else {
    const uint64_t* p = I.trees + 4 * (tree_offset(I.logn, k) + inner_offset(depth, level) + node);
    for (int j = 0; j < 4; j++) d[j] = p[j];
  }
}

// One value opening at byte offset `off`; returns its size.
__device__ uint64_t pcs_write_opening(const PcsInstance& I, uint32_t k, uint64_t idx, uint8_t* b, uint64_t off) {
  uint32_t depth = I.logn - k;
  uint4 v = I.layers[layer_offset(I.logn, k) + idx];
  pw64(b, off, idx);
  pw32(b, off + 8, v.x);
  pw32(b, off + 12, v.y);
  pw32(b, off + 16, v.z);
  pw32(b, off + 20, v.w);
  pw32(b, off + 24, depth);
  for (uint32_t l = 0; l < depth; l++) {
    uint64_t d[4];
    pcs_sibling(I, k, idx, l, d);
    pwdig(b, off + 28 + 32ull * l, d);
  }
  return opening_bytes(depth);
}

// One query (CircleFRIQueryV1 encoding: initial pair, layer count, then per layer
// its index, pair index and the left and right value openings) at byte `qoff` of
// `b`; the block's threads split the layers' openings.
__device__ void emit_query(const PcsInstance& I, uint64_t pair, uint8_t* b, uint64_t qoff) {
  const uint32_t R = I.rounds;
  if (threadIdx.x == 0) {
    pw64(b, qoff, pair);
    pw32(b, qoff + 8, R);
  }
  // thread (k, side) writes layer k's left (side 0) or right opening
  for (uint32_t t = threadIdx.x; t < 2 * R; t += blockDim.x) {
    uint32_t k = t >> 1, side = t & 1;
    uint64_t off = qoff + 12;
    for (uint32_t j = 0; j < k; j++) off += 12 + 2 * opening_bytes(I.logn - j);
    uint64_t pk = pair >> k;
    if (side == 0) {
      pw32(b, off, k);
      pw64(b, off + 4, pk);
    }
    uint64_t oo = off + 12 + (side ? opening_bytes(I.logn - k) : 0);
    pcs_write_opening(I, k, 2 * pk + side, b, oo);
  }
}

__global__ void pcs_emit_kernel(const PcsInstance* __restrict__ inst, const uint32_t* __restrict__ ids, uint32_t max_queries) {
  const PcsInstance& I = inst[ids[blockIdx.x]];
  uint8_t* b = I.proof;
  const uint32_t R = I.rounds;
  const uint64_t fcnt = 1ull << (I.logn - R);
  const uint64_t hdr = proof_header_bytes(R, fcnt);
  const uint64_t qbytes = proof_query_bytes(I.logn, R);
  const uint32_t q = blockIdx.y;
  if (q < I.queries) {
    emit_query(I, I.query_pairs[q], b, hdr + (uint64_t)q * qbytes);
    return;
  }
  if (q != max_queries) return;
  // header
  if (threadIdx.x == 0) {
    const uint8_t magic[8] = {0x41, 0x5a, 0x4b, 0x50, 0x46, 0x56, 0x31, 0x00};
    for (int i = 0; i < 8; i++) b[i] = magic[i];
    pw32(b, 8, 1);
    pw32(b, 12, 1);
    pw32(b, 16, 44);
    const uint8_t dm[8] = {0x41, 0x5a, 0x4b, 0x43, 0x44, 0x56, 0x31, 0x00};
    for (int i = 0; i < 8; i++) b[20 + i] = dm[i];
    pw32(b, 28, 1);
    pw32(b, 32, kP);
    pw32(b, 36, 31);
    pw32(b, 40, 2);
    pw32(b, 44, 1268011823u);
    pw32(b, 48, I.logn);
    pw32(b, 52, (uint32_t)((1ull << (31 - (I.logn + 1))) & 0x7FFFFFFFu));
    pw32(b, 56, I.logn - 1);
    pw32(b, 60, 1);
    pw32(b, 64, I.log_blowup);
    pw32(b, 68, I.queries);
    pw32(b, 72, 1);
    pw32(b, 76, I.grinding_bits);
    pw32(b, 80, 32);
    for (int k = 0; k < 4; k++) pw64(b, 84 + 8 * k, I.pub[k]);
    pw32(b, 116, R);
  }
  for (uint32_t r = threadIdx.x; r < R; r += blockDim.x) {
    uint64_t d[4];
    for (int k = 0; k < 4; k++) d[k] = I.commitments[4 * r + k];
    pwdig(b, 120 + 32ull * r, d);
  }
  const uint64_t foff = 120 + 32ull * R;
  if (threadIdx.x == 0) pw64(b, foff, fcnt);
  const uint4* fl = I.layers + layer_offset(I.logn, R);
  for (uint64_t i = threadIdx.x; i < fcnt; i += blockDim.x) {
    uint4 v = fl[i];
    pw32(b, foff + 8 + 16 * i, v.x);
    pw32(b, foff + 12 + 16 * i, v.y);
    pw32(b, foff + 16 + 16 * i, v.z);
    pw32(b, foff + 20 + 16 * i, v.w);
  }
  if (threadIdx.x == 0) pw32(b, foff + 8 + 16 * fcnt, I.queries);
  uint64_t tail = hdr + (uint64_t)I.queries * qbytes;
  if (I.n_claimed || I.has_nonce) {
    if (threadIdx.x == 0) pw32(b, tail, I.n_claimed);
    for (uint32_t c = threadIdx.x; c < I.n_claimed; c += blockDim.x)
      pcs_write_opening(I, 0, I.claimed[c], b, tail + 4 + (uint64_t)c * opening_bytes(I.logn));
    tail += 4 + (uint64_t)I.n_claimed * opening_bytes(I.logn);
  }
  if (I.has_nonce && threadIdx.x == 0) pw64(b, tail, I.nonce);
}

cudaError_t launch_pcs_emit(PcsInstance* d_inst, const uint32_t* d_ids, uint32_t nids, uint32_t max_queries, cudaStream_t s) {
  if (!nids) return cudaSuccess;
  dim3 grid(nids, max_queries + 1);
  pcs_emit_kernel<<<grid, 64, 0, s>>>(d_inst, d_ids, max_queries);
  return cudaGetLastError();
}

// Queries of committed resident layers (CircleFRIResidentQueryExtractorV1.extractQueries,
// CircleFRIFoldPlan.swift:1065-1148): block q writes query q, openings read from
// the layers and their resident trees, at byte q * (bytes per query) of `out`.
__global__ void query_extract_kernel(const PcsInstance* __restrict__ inst, const uint32_t* __restrict__ pairs, uint8_t* __restrict__ out) {
  const PcsInstance& I = *inst;
  emit_query(I, pairs[blockIdx.x], out, (uint64_t)blockIdx.x * proof_query_bytes(I.logn, I.rounds));
}

cudaError_t launch_query_extract(const PcsInstance* d_inst, const uint32_t* d_pairs, uint32_t count, uint8_t* d_out, cudaStream_t s) {
  if (!count) return cudaSuccess;
  query_extract_kernel<<<count, 64, 0, s>>>(d_inst, d_pairs, d_out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// QM31 fold-chain transcript (QM31FRIFold.swift:91-125, 769-862)
// ---------------------------------------------------------------------------
__global__ void qm31_prefix_kernel(Transcript* t, uint64_t input_count, uint32_t rounds) {
  if (threadIdx.x || blockIdx.x) return;
  Transcript s;
  tr_reset(s);
  FrameBuf f;
  qm31_frame(f, 0);
  fb_u64(f, input_count);
  fb_u32(f, rounds);
  fb_u32(f, kP);
  fb_u32(f, 4);
  fb_u32(f, 32);
  tr_absorb(s, f.b, f.n);
  *t = s;
}

cudaError_t launch_qm31_transcript_prefix(Transcript* d_t, uint64_t input_count, uint32_t rounds, cudaStream_t s) {
  qm31_prefix_kernel<<<1, 1, 0, s>>>(d_t, input_count, rounds);
  return cudaGetLastError();
}

// Challenges from caller-supplied commitments: kind 1 = Circle V1 rounds (prefix
// already absorbed), kind 2 = QM31 fold-chain rounds.
__global__ void transcript_rounds_kernel(Transcript* t, uint32_t kind, const uint64_t* roots, uint32_t rounds, uint64_t input_count, uint32_t* ch) {
  if (threadIdx.x || blockIdx.x) return;
  Transcript s = *t;
  uint64_t cnt = input_count;
  for (uint32_t r = 0; r < rounds; r++) {
    uint64_t root[4] = {roots[4 * r], roots[4 * r + 1], roots[4 * r + 2], roots[4 * r + 3]};
    uint32_t c[4];
    if (kind == kRootCircleRound)
      circle_round(s, r, root, c);
    else
      qm31_round(s, r, cnt, root, c);
    for (int k = 0; k < 4; k++) ch[4 * r + k] = c[k];
    cnt >>= 1;
  }
  *t = s;
}

cudaError_t launch_transcript_rounds_given(Transcript* d_t, uint32_t kind, const uint64_t* d_roots, uint32_t rounds, uint64_t input_count,
                                           uint32_t* d_ch, cudaStream_t s) {
  transcript_rounds_kernel<<<1, 1, 0, s>>>(d_t, kind, d_roots, rounds, input_count, d_ch);
  return cudaGetLastError();
}

// Canonicality gate (QM31CanonicalityCheck.swift:11-117; Metal :1668-1689):
// any limb >= p raises the flag.
__global__ void check_canonical_kernel(const uint32_t* __restrict__ w, uint64_t n, uint32_t* flag) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  for (; i < n; i += (uint64_t)gridDim.x * blockDim.x) bad |= w[i] >= kP;
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// Input scan of `count` QM31 coefficients: the canonicality gate, and whether any
// b, c or d limb is nonzero (then the coefficients are not a lifted M31
// polynomial and info->m31 is cleared).
__global__ void scan_input_kernel(const uint4* __restrict__ in, uint64_t count, uint32_t* bad, InputInfo* info) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool b = false, upper = false;
  for (; i < count; i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 v = in[i];
    b |= v.x >= kP || v.y >= kP || v.z >= kP || v.w >= kP;
    upper |= (v.y | v.z | v.w) != 0;
  }
  if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
  if (info && __any_sync(0xffffffffu, upper) && (threadIdx.x & 31) == 0) atomicAnd(&info->m31, 0u);
}

cudaError_t launch_scan_input(const uint4* d_in, uint64_t count, uint32_t* d_bad, InputInfo* d_info, cudaStream_t s) {
  if (!count) return cudaSuccess;
  uint64_t blocks = (count + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  scan_input_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_in, count, d_bad, d_info);
  return cudaGetLastError();
}

// One launch over many buffers: blockIdx.y picks the buffer (plus `base`), the
// blocks along x stride through its coefficients, checking [0, count) and
// writing zeros over [count, n).  One launch instead of a memset per buffer
// matters when another prover's superstep holds the GPU: every separate small
// launch waits for free SM slots between that superstep's large launches.
__global__ void scan_inputs_kernel(const ScanJob* __restrict__ jobs, uint32_t base, uint32_t* bad) {
  const ScanJob j = jobs[base + blockIdx.y];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool b = false, upper = false;
  for (uint64_t i = i0; i < j.count; i += stride) {
    uint4 v = j.in[i];
    b |= v.x >= kP || v.y >= kP || v.z >= kP || v.w >= kP;
    upper |= (v.y | v.z | v.w) != 0;
  }
  for (uint64_t i = j.count + i0; i < j.n; i += stride) j.in[i] = make_uint4(0u, 0u, 0u, 0u);
  if (__any_sync(0xffffffffu, b) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
  if (j.info && __any_sync(0xffffffffu, upper) && (threadIdx.x & 31) == 0) atomicAnd(&j.info->m31, 0u);
}

cudaError_t launch_scan_inputs(const ScanJob* d_jobs, uint32_t njobs, uint64_t max_n, uint32_t* d_bad, cudaStream_t s) {
  if (!njobs || !max_n) return cudaSuccess;
  uint64_t bx = (max_n + 255) / 256;
  if (bx > 64) bx = 64;
  for (uint32_t base = 0; base < njobs; base += 65535) {
    const uint32_t ny = njobs - base < 65535 ? njobs - base : 65535;
    scan_inputs_kernel<<<dim3((unsigned)bx, ny), 256, 0, s>>>(d_jobs, base, d_bad);
  }
  return cudaGetLastError();
}

cudaError_t launch_check_canonical(const uint32_t* d_words, uint64_t nwords, uint32_t* d_flag, cudaStream_t s) {
  if (!nwords) return cudaSuccess;
  uint64_t blocks = (nwords + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  check_canonical_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_words, nwords, d_flag);
  return cudaGetLastError();
}

}  // namespace azk
