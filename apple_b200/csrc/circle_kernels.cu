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
// Domain tables.  tw[off(s) + h] = stage-s FFT twiddle of block h, with
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

// Shared-memory tile layout: the four limbs of the tile's QM31 values as four u32
// arrays (an M31 tile uses only the first), then the tile's stage twiddles.  Stage
// j of the pass (global stage s_lo + j) pairs local indices differing in bit j + c,
// and its twiddle is tw[off(s) + (gi >> (s + 1))] = tw[off(s) + (hi << (m-1-j)) +
// (row >> (j + 1))]: 2^(m-1-j) consecutive table entries per tile, staged at
// stw + 2^m - 2^(m-j).
__device__ __forceinline__ uint32_t fft_stw_offset(uint32_t m, uint32_t j) { return (1u << m) - (1u << (m - j)); }

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

template <int THREADS>
__global__ void __launch_bounds__(THREADS) fft_pass_kernel(const FftJob* __restrict__ jobs, const uint2* __restrict__ work) {
  extern __shared__ uint32_t fsm[];
  const uint2 w = work[blockIdx.x];
  const FftJob& job = jobs[w.x];
  const uint32_t logn = job.logn;
  const FftPassGeom g = fft_pass_geom(logn, job.pass);
  const uint32_t T = 1u << (g.m + g.c);
  const uint64_t N = 1ull << logn;
  const bool first = job.pass == 0;
  const bool last = job.pass == fft_high_chunks(logn);
  const InputInfo* info = job.info;
  const bool narrow = info != nullptr && job.narrow != nullptr && info->m31 != 0;
  const uint64_t count = (info != nullptr && info->count != 0) ? info->count : N;
  uint32_t* sa = fsm;
  uint32_t* sb = sa + T;
  uint32_t* sc = sb + T;
  uint32_t* sd = sc + T;
  uint32_t* stw = sd + T;

  // this tile's twiddles, one coalesced run per stage
  const uint32_t midbits = g.s_lo > g.c ? g.s_lo - g.c : 0;
  const uint64_t hi = (uint64_t)w.y >> midbits;
  for (uint32_t j = 0; j < g.m; j++) {
    const uint32_t cnt = 1u << (g.m - 1 - j);
    const uint32_t* src = job.tw + tw_offset(logn, g.s_lo + j) + (hi << (g.m - 1 - j));
    uint32_t* dst = stw + fft_stw_offset(g.m, j);
    for (uint32_t r = threadIdx.x; r < cnt; r += THREADS) dst[r] = __ldg(src + r);
  }
  // the tile (the first pass skips coefficients known to be zero)
  for (uint32_t L = threadIdx.x; L < T; L += THREADS) {
    const uint64_t gi = fft_global_index(g, w.y, L);
    if (narrow) {
      uint32_t v;
      if (first)
        v = gi < count ? __ldg(reinterpret_cast<const uint32_t*>(job.in) + 4 * gi) : 0u;
      else
        v = job.narrow[gi];
      sa[L] = v;
    } else {
      uint4 v;
      if (first)
        v = gi < count ? __ldg(job.in + gi) : make_uint4(0u, 0u, 0u, 0u);
      else
        v = job.out[gi];
      sa[L] = v.x;
      sb[L] = v.y;
      sc[L] = v.z;
      sd[L] = v.w;
    }
  }
  __syncthreads();

  // stages two at a time (radix 4 in registers), then one more if m is odd
  int j = (int)g.m - 1;
  for (; j >= 1; j -= 2) {
    const uint32_t p = (uint32_t)j + g.c;  // stage j pairs bit p, stage j-1 pairs bit p-1
    const uint32_t* tw_j = stw + fft_stw_offset(g.m, (uint32_t)j);
    const uint32_t* tw_j1 = stw + fft_stw_offset(g.m, (uint32_t)j - 1);
    const uint32_t lowmask = (1u << (p - 1)) - 1;
    for (uint32_t k = threadIdx.x; k < T / 4; k += THREADS) {
      const uint32_t e0 = ((k & ~lowmask) << 2) | (k & lowmask);
      const uint32_t e1 = e0 | (1u << (p - 1)), e2 = e0 | (1u << p), e3 = e2 | (1u << (p - 1));
      const uint32_t row = e0 >> g.c;
      const uint32_t t1 = tw_j[row >> (j + 1)];
      const uint32_t t2a = tw_j1[row >> j], t2b = tw_j1[(row >> j) | 1u];
      if (narrow) {
        uint32_t v0 = sa[e0], v1 = sa[e1], v2 = sa[e2], v3 = sa[e3];
        bfly_m31(v0, v2, t1);
        bfly_m31(v1, v3, t1);
        bfly_m31(v0, v1, t2a);
        bfly_m31(v2, v3, t2b);
        sa[e0] = v0;
        sa[e1] = v1;
        sa[e2] = v2;
        sa[e3] = v3;
      } else {
        qm31 v0 = {sa[e0], sb[e0], sc[e0], sd[e0]}, v1 = {sa[e1], sb[e1], sc[e1], sd[e1]};
        qm31 v2 = {sa[e2], sb[e2], sc[e2], sd[e2]}, v3 = {sa[e3], sb[e3], sc[e3], sd[e3]};
        bfly_q(v0, v2, t1);
        bfly_q(v1, v3, t1);
        bfly_q(v0, v1, t2a);
        bfly_q(v2, v3, t2b);
        sa[e0] = v0.a, sb[e0] = v0.b, sc[e0] = v0.c, sd[e0] = v0.d;
        sa[e1] = v1.a, sb[e1] = v1.b, sc[e1] = v1.c, sd[e1] = v1.d;
        sa[e2] = v2.a, sb[e2] = v2.b, sc[e2] = v2.c, sd[e2] = v2.d;
        sa[e3] = v3.a, sb[e3] = v3.b, sc[e3] = v3.c, sd[e3] = v3.d;
      }
    }
    __syncthreads();
  }
  if (j == 0) {
    const uint32_t p = g.c;
    for (uint32_t k = threadIdx.x; k < T / 2; k += THREADS) {
      const uint32_t L = ((k >> p) << (p + 1)) | (k & ((1u << p) - 1));
      const uint32_t R = L | (1u << p);
      const uint32_t t = stw[(L >> g.c) >> 1];
      if (narrow) {
        uint32_t l = sa[L], r = sa[R];
        bfly_m31(l, r, t);
        sa[L] = l;
        sa[R] = r;
      } else {
        qm31 l = {sa[L], sb[L], sc[L], sd[L]}, r = {sa[R], sb[R], sc[R], sd[R]};
        bfly_q(l, r, t);
        sa[L] = l.a, sb[L] = l.b, sc[L] = l.c, sd[L] = l.d;
        sa[R] = r.a, sb[R] = r.b, sc[R] = r.c, sd[R] = r.d;
      }
    }
    __syncthreads();
  }

  for (uint32_t L = threadIdx.x; L < T; L += THREADS) {
    const uint64_t gi = fft_global_index(g, w.y, L);
    if (!narrow)
      job.out[gi] = make_uint4(sa[L], sb[L], sc[L], sd[L]);
    else if (last)
      job.out[gi] = make_uint4(sa[L], 0u, 0u, 0u);
    else
      job.narrow[gi] = sa[L];
  }
}

// four limb arrays of 4096 values + 4095 staged twiddles
static constexpr size_t kFftSmem = ((size_t)16 << kFftLowBits) + ((size_t)4 << kFftLowBits);
static constexpr int kFftThreads = 512;

cudaError_t prepare_fft_kernels() {
  return cudaFuncSetAttribute(fft_pass_kernel<kFftThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFftSmem);
}

cudaError_t launch_fft_pass(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s) {
  if (nwork == 0) return cudaSuccess;
  fft_pass_kernel<kFftThreads><<<nwork, kFftThreads, kFftSmem, s>>>(d_jobs, d_work);
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
__global__ void fold_qm31_inv_kernel(const uint4* __restrict__ prev, const uint4* __restrict__ inv, const uint32_t* __restrict__ chp, uint4* __restrict__ out,
                                     uint64_t n_out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_out) return;
  qm31 ch = {__ldcg(chp), __ldcg(chp + 1), __ldcg(chp + 2), __ldcg(chp + 3)};
  uint4 p = prev[2 * i], q = prev[2 * i + 1], t = inv[i];
  qm31 pos = {p.x, p.y, p.z, p.w}, neg = {q.x, q.y, q.z, q.w};
  qm31 odd = q_mul(q_sub(pos, neg), qm31{t.x, t.y, t.z, t.w});
  qm31 r = q_half(q_add(q_add(pos, neg), q_mul(ch, odd)));
  out[i] = make_uint4(r.a, r.b, r.c, r.d);
}

cudaError_t launch_fold_qm31_inv(const uint4* prev, const uint4* inv, const uint32_t* ch, uint4* out, uint64_t n_out, cudaStream_t s) {
  if (n_out == 0) return cudaSuccess;
  fold_qm31_inv_kernel<<<(unsigned)((n_out + 255) / 256), 256, 0, s>>>(prev, inv, ch, out, n_out);
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

__global__ void pcs_emit_kernel(const PcsInstance* __restrict__ inst, const uint32_t* __restrict__ ids, uint32_t max_queries) {
  const PcsInstance& I = inst[ids[blockIdx.x]];
  uint8_t* b = I.proof;
  const uint32_t R = I.rounds;
  const uint64_t fcnt = 1ull << (I.logn - R);
  const uint64_t hdr = proof_header_bytes(R, fcnt);
  const uint64_t qbytes = proof_query_bytes(I.logn, R);
  const uint32_t q = blockIdx.y;
  if (q < I.queries) {
    uint64_t qoff = hdr + (uint64_t)q * qbytes;
    uint64_t pair = I.query_pairs[q];
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

cudaError_t launch_check_canonical(const uint32_t* d_words, uint64_t nwords, uint32_t* d_flag, cudaStream_t s) {
  if (!nwords) return cudaSuccess;
  uint64_t blocks = (nwords + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  check_canonical_kernel<<<(unsigned)blocks, 256, 0, s>>>(d_words, nwords, d_flag);
  return cudaGetLastError();
}

}  // namespace azk
