// One-limb Circle FFT passes for transforms of 2^12 values or more whose inputs
// are lifted M31 polynomials (b = c = d = 0 in every coefficient, hence in every
// intermediate value): the FFT of CircleCodeword.swift:72-98 (Metal
// HashMerkleKernels.metal:1881-1908), run as register-blocked radix-16 tiles.
//
// Tile: 4096 values, local index L (12 bits) = (row << c) | col, where the m row
// bits are the pass's stages (global stage s_lo + j pairs row bit j) and the c =
// 12 - m column bits are the lowest global index bits (contiguous in memory).
// The 256 threads of a CTA hold 16 values each, and a tile runs in three
// sub-passes; sub-pass q gives each thread the 16 values that differ in L bits
// 4q ... 4q + 3 and runs the butterflies of the stages among those bits in
// registers (radix 16: four stages, 32 butterflies, one twiddle vector load per
// stage).  Between sub-passes the values go through one shared 16 KB buffer whose
// XOR swizzle makes every access pattern of the three sub-passes free of bank
// conflicts (the last sub-pass reads and writes 16-byte vectors).  Twiddles come
// straight from the domain table: the 2^(3-k) twiddles of the stage on owned bit
// k are consecutive table entries, loaded as one vector.
//
// Kernels:
//  - fft_m31_tile_kernel: one CTA per tile.  First passes read the a limbs of the
//    QM31 coefficients (only the nonzero prefix), later high-stage passes the
//    one-word exchange buffer; the pass writes the exchange buffer, or the QM31
//    codeword when it is the transform's only pass (log 12).
//  - fft_m31_low_tma_kernel: the low-stage (last) pass of transforms above 2^12,
//    persistent.  Each CTA walks the work list; its tile's 16 KB of input is one
//    contiguous run of the exchange buffer, copied into shared memory by one bulk
//    copy (cp.async.bulk, completion counted on an mbarrier) that is issued for the
//    next tile as soon as the current tile's first sub-pass has read its copy, so
//    the load runs under the remaining sub-passes.  Every wait on the mbarrier is
//    bounded: a wait that runs out raises `status`, and the CTA returns after one
//    more bounded wait for the copy it was waiting on.
//  - fft_q_tile_kernel: the same tiles over QM31 values (inputs that are not lifted
//    M31 polynomials), in place in the codeword buffer between passes.
#include "azk_bulk.cuh"
#include "azk_field.cuh"
#include "azk_internal.h"

namespace azk {

namespace {

constexpr uint32_t kTile = 1u << kFftLowBits;  // 4096 values
constexpr int kThreads = 256;

__device__ __forceinline__ uint64_t twoff(uint32_t logn, uint32_t s) {
  const uint64_t n = 1ull << logn;
  return n - (n >> s);
}

// Bank-conflict-free placement of tile value L in the shared buffer: bits 2, 3 and
// 4 are flipped by bits 5, 6 and 8.  Sub-pass 2 (owned bits 8-11, a warp spans L
// bits 0-4), sub-pass 1 (owned bits 4-7, a warp spans L bits 0-3 and 8) and the
// vector accesses of sub-pass 0 (owned bits 0-3; a quarter warp spans L bits 4-6)
// each reach 32 distinct banks; bits 0 and 1 are never moved, so four consecutive
// values stay one aligned 16-byte vector.
__device__ __forceinline__ uint32_t swz(uint32_t L) { return L ^ (((L >> 3) & 12u) | ((L >> 4) & 16u)); }

// The doubled twiddle table (2 t at tw + N): the butterflies multiply by 2t.
__device__ __forceinline__ const uint32_t* tw2(const FftJob& job) { return job.tw + (1ull << job.logn); }

// (l, r) -> (l + r t, l - r t), given t2 = 2t
__device__ __forceinline__ void bfly(uint32_t& l, uint32_t& r, uint32_t t2) {
  const uint32_t rt = m31_mul_dbl(r, t2);
  const uint32_t a = m31_add(l, rt);
  r = m31_sub(l, rt);
  l = a;
}

// The 2^R consecutive twiddles at `p` (R = 0..3), aligned to their count.
template <int R>
__device__ __forceinline__ void load_tw(const uint32_t* __restrict__ p, uint32_t (&t)[8]) {
  if constexpr (R == 0) {
    t[0] = __ldg(p);
  } else if constexpr (R == 1) {
    const uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
    t[0] = a.x, t[1] = a.y;
  } else if constexpr (R == 2) {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    t[0] = a.x, t[1] = a.y, t[2] = a.z, t[3] = a.w;
  } else {
    const uint4 a = __ldg(reinterpret_cast<const uint4*>(p));
    const uint4 b = __ldg(reinterpret_cast<const uint4*>(p) + 1);
    t[0] = a.x, t[1] = a.y, t[2] = a.z, t[3] = a.w, t[4] = b.x, t[5] = b.y, t[6] = b.z, t[7] = b.w;
  }
}

struct Pass {
  uint32_t logn, s_lo, m, c;
  uint64_t hi;     // tile bits above the pass's stages
  uint64_t gbase;  // global index of L = 0
  __device__ __forceinline__ uint64_t gidx(uint32_t L) const {
    return gbase | ((uint64_t)(L >> c) << s_lo) | (L & ((1u << c) - 1u));
  }
};

__device__ __forceinline__ Pass make_pass(const FftJob& job, uint64_t tile) {
  const FftPassGeom g0 = fft_pass_geom(job.logn, job.pass);
  Pass p;
  p.logn = job.logn;
  p.s_lo = g0.s_lo;
  p.m = g0.m;
  p.c = kFftLowBits - g0.m;
  const uint32_t midbits = p.s_lo - p.c;  // 0 for the low pass (s_lo = c = 0)
  const uint64_t mid = tile & ((1ull << midbits) - 1);
  p.hi = tile >> midbits;
  p.gbase = (p.hi << (p.s_lo + p.m)) | (mid << p.c);
  return p;
}

// The low-stage pass of a transform above 2^12 (s_lo = 0, m = 12, c = 0): the same
// geometry as make_pass, with the constants visible to the compiler.
__device__ __forceinline__ Pass low_pass(const FftJob& job, uint64_t tile) {
  Pass p;
  p.logn = job.logn;
  p.s_lo = 0;
  p.m = kFftLowBits;
  p.c = 0;
  p.hi = tile;
  p.gbase = tile << kFftLowBits;
  return p;
}

// The stage of sub-pass Q on owned bit K (L bit 4Q + K) over the thread's 16
// values v[b] (bit k of b = L bit 4Q + k; Lbase = the thread's L with those bits
// zero): 8 butterflies with the 2^(3-K) twiddles of the stage's blocks above it.
__device__ __forceinline__ void bfly(qm31& l, qm31& r, uint32_t t) {
  bfly(l.a, r.a, t);
  bfly(l.b, r.b, t);
  bfly(l.c, r.c, t);
  bfly(l.d, r.d, t);
}

// Twiddles of one sub-pass, loaded ahead of the butterflies that use them (before
// the barrier or bulk-copy wait that precedes the sub-pass, so their latency hides
// behind it): t[K] holds the 2^(3-K) twiddles of the stage on owned bit K.
struct TwSet {
  uint32_t t[4][8];
};

// Stage j = 4Q + K - c of the pass (global stage s_lo + j): its twiddles for the
// thread's values start at tw[off(s) + (hi << (m-1-j)) + ((Lbase >> c) >> (j+1))].
template <int Q, int K>
__device__ __forceinline__ void tw_stage(uint32_t Lbase, const Pass& p, const uint32_t* __restrict__ tw, uint32_t (&t)[8]) {
  const uint32_t j = 4 * Q + K - p.c;
  const uint32_t s = p.s_lo + j;
  const uint64_t base = twoff(p.logn, s) + (p.hi << (p.m - 1 - j)) + ((uint64_t)(Lbase >> p.c) >> (j + 1));
  load_tw<3 - K>(tw + base, t);
}

// The stages of sub-pass Q run from owned bit `kstart` down; owned bits below the
// pass's column count are columns (no butterflies, no twiddles).
template <int Q>
__device__ __forceinline__ void tw_load(TwSet& w, uint32_t Lbase, const Pass& p, const uint32_t* __restrict__ tw, int kstart) {
  if (kstart >= 3 && 4 * Q + 3 >= p.c) tw_stage<Q, 3>(Lbase, p, tw, w.t[3]);
  if (kstart >= 2 && 4 * Q + 2 >= p.c) tw_stage<Q, 2>(Lbase, p, tw, w.t[2]);
  if (kstart >= 1 && 4 * Q + 1 >= p.c) tw_stage<Q, 1>(Lbase, p, tw, w.t[1]);
  if (4 * Q >= p.c) tw_stage<Q, 0>(Lbase, p, tw, w.t[0]);
}

// The stage on owned bit K over the thread's 16 values v[b] (bit k of b = L bit
// 4Q + k): 8 butterflies with the 2^(3-K) twiddles of the stage's blocks above it.
template <int K, class V>
__device__ __forceinline__ void stage(V (&v)[16], const uint32_t (&t)[8]) {
#pragma unroll
  for (int b = 0; b < 16; b++) {
    if (b & (1 << K)) continue;
    bfly(v[b], v[b | (1 << K)], t[b >> (K + 1)]);
  }
}

template <int Q, class V>
__device__ __forceinline__ void subpass(V (&v)[16], const TwSet& w, const Pass& p, int kstart) {
  if (kstart >= 3 && 4 * Q + 3 >= p.c) stage<3>(v, w.t[3]);
  if (kstart >= 2 && 4 * Q + 2 >= p.c) stage<2>(v, w.t[2]);
  if (kstart >= 1 && 4 * Q + 1 >= p.c) stage<1>(v, w.t[1]);
  if (4 * Q >= p.c) stage<0>(v, w.t[0]);
}

// Sub-passes 1 and 0 after sub-pass 2 has left its values in `Y` (synchronised;
// `w1` holds sub-pass 1's twiddles, loaded before that barrier), then the pass's
// output: the exchange buffer (high-stage passes, from the last sub-pass that has
// stages) or the QM31 codeword (the transform's last pass, from `Y` in coalesced
// rows).  `last` passes have c = 0.
__device__ __forceinline__ uint32_t sub1_base(uint32_t t) { return (t & 15u) | ((t >> 4) << 8); }

__device__ __forceinline__ void finish_tile(uint32_t* Y, const FftJob& job, const Pass& p, bool last, const TwSet& w1) {
  const uint32_t t = threadIdx.x;
  uint32_t v[16];
  const uint32_t LB = sub1_base(t);
#pragma unroll
  for (int b = 0; b < 16; b++) v[b] = Y[swz(LB | ((uint32_t)b << 4))];
  subpass<1>(v, w1, p, 3);
  if (p.c >= 4) {  // no stages among L bits 0-3: the pass ends here (never the last pass)
#pragma unroll
    for (int b = 0; b < 16; b++) job.narrow[p.gidx(LB | ((uint32_t)b << 4))] = v[b];
    return;
  }
#pragma unroll
  for (int b = 0; b < 16; b++) Y[swz(LB | ((uint32_t)b << 4))] = v[b];
  const uint32_t LC = t << 4;
  TwSet w0;
  tw_load<0>(w0, LC, p, tw2(job), 3);
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const uint4 q = *reinterpret_cast<const uint4*>(Y + swz(LC | (4u * r)));
    v[4 * r] = q.x, v[4 * r + 1] = q.y, v[4 * r + 2] = q.z, v[4 * r + 3] = q.w;
  }
  subpass<0>(v, w0, p, 3);
  if (!last) {
    // c >= 2: four consecutive L are four consecutive, 16-byte aligned global words
#pragma unroll
    for (int r = 0; r < 4; r++)
      *reinterpret_cast<uint4*>(job.narrow + p.gidx(LC | (4u * r))) = make_uint4(v[4 * r], v[4 * r + 1], v[4 * r + 2], v[4 * r + 3]);
    return;
  }
#pragma unroll
  for (int r = 0; r < 4; r++) *reinterpret_cast<uint4*>(Y + swz(LC | (4u * r))) = make_uint4(v[4 * r], v[4 * r + 1], v[4 * r + 2], v[4 * r + 3]);
  __syncthreads();
#pragma unroll 4
  for (uint32_t r = 0; r < 16; r++) {
    const uint32_t L = t + kThreads * r;
    job.out[p.gbase + L] = make_uint4(Y[swz(L)], 0u, 0u, 0u);
  }
}

// make_pass with the pass's stage count M (> 0) known at compile time: the same
// values, so the sub-pass conditions and index arithmetic fold to constants.
template <int M>
__device__ __forceinline__ Pass make_pass_m(const FftJob& job, uint64_t tile) {
  Pass p = make_pass(job, tile);
  if constexpr (M > 0) {
    p.m = M;
    p.c = kFftLowBits - M;
  }
  return p;
}

template <int M>
__device__ __forceinline__ void m31_tile(const FftJob& job, uint2 w, uint32_t* Y) {
  const Pass p = make_pass_m<M>(job, w.y);
  const uint64_t N = 1ull << p.logn;
  const bool first = job.pass == 0;
  const bool last = job.pass == fft_high_chunks(p.logn);
  const uint64_t count = (job.info != nullptr && job.info->count != 0) ? job.info->count : N;
  // a first pass over a nonzero prefix of at most N/4 that holds the transform's
  // two top stages (m >= 2; they are L bits 11 and 10): every value with either of
  // those bits set is zero, so the two top stages only copy (l + 0 t, l - 0 t) and
  // only 4 of the thread's 16 values are read
  const bool top_zero = first && p.m >= 2 && count <= (N >> 2);
  const uint32_t t = threadIdx.x;
  const uint32_t LA = t;
  TwSet w2;
  tw_load<2>(w2, LA, p, tw2(job), top_zero ? 1 : 3);
  uint32_t v[16];
  if (first) {
    const uint32_t* in_a = reinterpret_cast<const uint32_t*>(job.in);
    if (top_zero) {
      uint32_t x[4];
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const uint64_t gi = p.gidx(LA | ((uint32_t)b << 8));
        x[b] = gi < count ? __ldg(in_a + 4 * gi) : 0u;
      }
#pragma unroll
      for (int b = 0; b < 16; b++) v[b] = x[b & 3];
    } else {
#pragma unroll
      for (int b = 0; b < 16; b++) {
        const uint64_t gi = p.gidx(LA | ((uint32_t)b << 8));
        v[b] = gi < count ? __ldg(in_a + 4 * gi) : 0u;
      }
    }
  } else {
#pragma unroll
    for (int b = 0; b < 16; b++) v[b] = __ldg(job.narrow + p.gidx(LA | ((uint32_t)b << 8)));
  }
  subpass<2>(v, w2, p, top_zero ? 1 : 3);
  if (p.c >= 8) {  // every stage among L bits 8-11 (a high-stage pass of at most 4 stages)
#pragma unroll
    for (int b = 0; b < 16; b++) job.narrow[p.gidx(LA | ((uint32_t)b << 8))] = v[b];
    return;
  }
#pragma unroll
  for (int b = 0; b < 16; b++) Y[swz(LA | ((uint32_t)b << 8))] = v[b];
  TwSet w1;
  tw_load<1>(w1, sub1_base(t), p, tw2(job), 3);
  __syncthreads();
  finish_tile(Y, job, p, last, w1);
}

// One CTA per tile; the passes that hold most of the values of large transforms
// (6 to 10 high stages, and the single pass of a 2^12 transform) run code
// specialised for their stage count, the others the general form.
__global__ void __launch_bounds__(kThreads, 4) fft_m31_tile_kernel(const FftJob* __restrict__ jobs, const uint2* __restrict__ work) {
  __shared__ __align__(16) uint32_t Y[kTile];
  const uint2 w = work[blockIdx.x];
  const FftJob& job = jobs[w.x];
  switch (fft_pass_geom(job.logn, job.pass).m) {
    case 10: m31_tile<10>(job, w, Y); break;
    case 9: m31_tile<9>(job, w, Y); break;
    case 8: m31_tile<8>(job, w, Y); break;
    case 7: m31_tile<7>(job, w, Y); break;
    case 6: m31_tile<6>(job, w, Y); break;
    case 12: m31_tile<12>(job, w, Y); break;
    default: m31_tile<0>(job, w, Y); break;
  }
}

// ---------------------------------------------------------------------------
// Four-limb (QM31) tiles for transforms of 2^12 values or more whose inputs are
// not lifted M31 polynomials: the same sub-passes over 16-byte values.  The
// shared buffer holds 4096 values (64 KB) placed by swq, which flips bits 0-2 by
// bits 4-6, so the 16-byte accesses of all three sub-passes (a quarter warp spans
// L bits 0-2 in sub-passes 2 and 1 and bits 4-6 in sub-pass 0) fall in 8 distinct
// 16-byte bank groups.  The first pass reads the coefficients (the nonzero prefix)
// and writes the codeword buffer; later passes read and write it in place (each
// tile only its own values).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t swq(uint32_t L) { return L ^ ((L >> 4) & 7u); }
__device__ __forceinline__ qm31 to_q(uint4 v) { return qm31{v.x, v.y, v.z, v.w}; }
__device__ __forceinline__ uint4 from_q(qm31 v) { return make_uint4(v.a, v.b, v.c, v.d); }

__global__ void __launch_bounds__(kThreads, 2) fft_q_tile_kernel(const FftJob* __restrict__ jobs, const uint2* __restrict__ work) {
  extern __shared__ __align__(16) uint4 Yq[];  // kTile values
  const uint2 w = work[blockIdx.x];
  const FftJob& job = jobs[w.x];
  const Pass p = make_pass(job, w.y);
  const uint64_t N = 1ull << p.logn;
  const bool first = job.pass == 0;
  const bool last = job.pass == fft_high_chunks(p.logn);
  const uint64_t count = (job.info != nullptr && job.info->count != 0) ? job.info->count : N;
  const bool top_zero = first && p.m >= 2 && count <= (N >> 2);
  const uint32_t t = threadIdx.x;
  const uint32_t LA = t;
  TwSet tws;
  tw_load<2>(tws, LA, p, tw2(job), top_zero ? 1 : 3);
  qm31 v[16];
  if (first) {
    const int loads = top_zero ? 4 : 16;
#pragma unroll
    for (int b = 0; b < 16; b++) {
      if (b >= loads) {
        v[b] = v[b & 3];
        continue;
      }
      const uint64_t gi = p.gidx(LA | ((uint32_t)b << 8));
      v[b] = gi < count ? to_q(__ldg(job.in + gi)) : qm31{0u, 0u, 0u, 0u};
    }
  } else {
#pragma unroll
    for (int b = 0; b < 16; b++) v[b] = to_q(job.out[p.gidx(LA | ((uint32_t)b << 8))]);
  }
  subpass<2>(v, tws, p, top_zero ? 1 : 3);
  if (p.c >= 8) {
#pragma unroll
    for (int b = 0; b < 16; b++) job.out[p.gidx(LA | ((uint32_t)b << 8))] = from_q(v[b]);
    return;
  }
#pragma unroll
  for (int b = 0; b < 16; b++) Yq[swq(LA | ((uint32_t)b << 8))] = from_q(v[b]);
  const uint32_t LB = sub1_base(t);
  tw_load<1>(tws, LB, p, tw2(job), 3);
  __syncthreads();
#pragma unroll
  for (int b = 0; b < 16; b++) v[b] = to_q(Yq[swq(LB | ((uint32_t)b << 4))]);
  subpass<1>(v, tws, p, 3);
  if (p.c >= 4) {
#pragma unroll
    for (int b = 0; b < 16; b++) job.out[p.gidx(LB | ((uint32_t)b << 4))] = from_q(v[b]);
    return;
  }
#pragma unroll
  for (int b = 0; b < 16; b++) Yq[swq(LB | ((uint32_t)b << 4))] = from_q(v[b]);
  const uint32_t LC = t << 4;
  tw_load<0>(tws, LC, p, tw2(job), 3);
  __syncthreads();
#pragma unroll
  for (int b = 0; b < 16; b++) v[b] = to_q(Yq[swq(LC | (uint32_t)b)]);
  subpass<0>(v, tws, p, 3);
  if (!last) {
#pragma unroll
    for (int b = 0; b < 16; b++) job.out[p.gidx(LC | (uint32_t)b)] = from_q(v[b]);
    return;
  }
  // the last pass (c = 0): coalesced rows through the shared buffer
#pragma unroll
  for (int b = 0; b < 16; b++) Yq[swq(LC | (uint32_t)b)] = from_q(v[b]);
  __syncthreads();
#pragma unroll 4
  for (uint32_t r = 0; r < 16; r++) {
    const uint32_t L = t + kThreads * r;
    job.out[p.gbase + L] = Yq[swq(L)];
  }
}

// Queue the bulk copy of work item `item`'s input tile (4096 contiguous words of the
// exchange buffer: the low pass has c = 0 and s_lo = 0, so tile w is words
// [4096 w, 4096 w + 4096); 16 KB, 16-byte aligned) into X.
__device__ __forceinline__ void fetch_low_tile(const FftJob* __restrict__ jobs, uint2 w, uint32_t* X, uint64_t* bar) {
  const FftJob& job = jobs[w.x];
  mbar_expect_tx(bar, kTile * 4);
  bulk_copy_g2s(X, job.narrow + ((uint64_t)w.y << kFftLowBits), kTile * 4, bar);
}

__global__ void __launch_bounds__(kThreads, 4) fft_m31_low_tma_kernel(const FftJob* __restrict__ jobs, const uint2* __restrict__ work, uint32_t nwork,
                                                                      uint32_t* __restrict__ status) {
  __shared__ __align__(128) uint32_t X[kTile];  // bulk-copy landing buffer (linear)
  __shared__ __align__(16) uint32_t Y[kTile];   // swizzled working buffer
  __shared__ __align__(8) uint64_t bar;
  const uint32_t t = threadIdx.x;
  uint32_t item = blockIdx.x;
  if (item >= nwork) return;
  if (t == 0) {
    mbar_init(&bar, 1);
    fetch_low_tile(jobs, work[item], X, &bar);
  }
  __syncthreads();
  uint32_t phase = 0;
  for (; item < nwork; item += gridDim.x) {
    const uint2 w = work[item];
    const FftJob& job = jobs[w.x];
    const Pass p = low_pass(job, w.y);
    TwSet w2;
    tw_load<2>(w2, t, p, tw2(job), 3);
    const bool ok = mbar_wait(&bar, phase);
    phase ^= 1u;
    uint32_t v[16];
#pragma unroll
    for (int b = 0; b < 16; b++) v[b] = X[t + kThreads * b];
    subpass<2>(v, w2, p, 3);
#pragma unroll
    for (int b = 0; b < 16; b++) Y[swz(t | ((uint32_t)b << 8))] = v[b];
    TwSet w1;
    tw_load<1>(w1, sub1_base(t), p, tw2(job), 3);
    // X has been read by every thread: the next tile's copy may land in it
    if (__syncthreads_or(!ok)) {
      // the copy that did not complete may still land: wait for it once more
      // (bounded) before the CTA gives up its shared memory
      if (t == 0) {
        atomicOr(status, 1u);
        mbar_wait(&bar, phase ^ 1u);
      }
      return;
    }
    const uint32_t next = item + gridDim.x;
    if (t == 0 && next < nwork) {
      fence_proxy_async_smem();
      fetch_low_tile(jobs, work[next], X, &bar);
    }
    finish_tile(Y, job, p, true, w1);
    __syncthreads();  // Y is rewritten by the next tile's first sub-pass
  }
}

int g_low_grid[64] = {0};  // resident CTAs of the persistent kernel, per device

}  // namespace

cudaError_t prepare_fft_m31_kernels() {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaFuncSetAttribute(fft_q_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kTile * sizeof(uint4)));
  if (e != cudaSuccess) return e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_m31_low_tma_kernel, kThreads, 0)) != cudaSuccess) return e;
  if (dev >= 0 && dev < 64) g_low_grid[dev] = sms * (per_sm > 0 ? per_sm : 1);
  return cudaSuccess;
}

cudaError_t launch_fft_m31_tiles(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s) {
  if (nwork == 0) return cudaSuccess;
  fft_m31_tile_kernel<<<nwork, kThreads, 0, s>>>(d_jobs, d_work);
  return cudaGetLastError();
}

cudaError_t launch_fft_q_tiles(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s) {
  if (nwork == 0) return cudaSuccess;
  fft_q_tile_kernel<<<nwork, kThreads, kTile * sizeof(uint4), s>>>(d_jobs, d_work);
  return cudaGetLastError();
}

cudaError_t launch_fft_m31_low(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t* d_status, cudaStream_t s) {
  if (nwork == 0) return cudaSuccess;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
  const uint32_t resident = (uint32_t)g_low_grid[dev];
  const uint32_t grid = resident && resident < nwork ? resident : nwork;
  fft_m31_low_tma_kernel<<<grid, kThreads, 0, s>>>(d_jobs, d_work, nwork, d_status);
  return cudaGetLastError();
}

}  // namespace azk
