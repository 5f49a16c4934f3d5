// M31 multilinear sum-check prover on the device (M31MultilinearSumcheckProofBuilderV1,
// SumcheckOracle.swift:797-868; statement digest :743-754; word digest :1288-1299;
// transcript frames :1066-1106).
//
// A table is proved by one group of warps: one warp computes the statement's word
// digest, a sequential sponge over the whole table (about 30,000 dependent
// permutations for 2^20 words), while the group's other warps sum the table for
// round 0; then the group proves the rounds.  A table of 2^20 words is 4 MiB, so
// each round is a few microseconds of one SM, and keeping a table in one group
// needs no grid-wide wait.  The single-table kernel is one CTA of 8 warps; the
// batched kernel packs four tables into one CTA (sumcheck_packed_kernel).
#include "azk_field.cuh"
#include "azk_internal.h"

namespace azk {

__device__ void sc_frame(FrameBuf& f, uint8_t type) {
  const char dom[] = "AppleZKProver.M31MultilinearSumcheck";
  f.n = 0;
  fb_u32(f, 36);
  fb_str(f, dom, 36);
  fb_u32(f, 1);
  fb_u8(f, type);
}

// ---------------------------------------------------------------------------
// Keccak-f[1600] spread over one warp, for the statement digest: one sponge over
// the whole table is a chain of ~30,000 dependent permutations, so what counts is
// the latency of one permutation, not throughput.  Lane x + 5y (< 25) holds state
// lane (x, y); lanes 25..31 follow lane 0's indices and store nothing.  A round
// is two exchanges, and its cost follows the number of exchange instructions
// more than the number of dependent stages (measured on B200: three shuffle
// stages 2.43 us per permutation, two shuffle stages 2.30 us, this form 1.98 us):
//   1. every lane stores its lane into a column-major shared array (columns
//      padded to 6 words so a column is two 16-byte loads and one 8-byte load)
//      and reads columns x - 1 and x + 1: theta's D[x], then rho's rotation of
//      its own lane, e = rotl(a ^ D[x], rho[x, y]), at the source.  Rounds
//      alternate between two arrays, so the one __syncwarp after the stores also
//      orders the previous round's loads of the other array before its next stores;
//   2. pi and chi in one gather: lane (x, y) shuffles e from the pi sources of
//      (x, y), (x + 1, y) and (x + 2, y); iota enters as chi(b0 ^ rc, b1, b2)
//      (= chi(b0, b1, b2) ^ rc) through a mask that is zero except on lane 0, so
//      its XOR overlaps the wait for the later shuffles.
// ---------------------------------------------------------------------------
__constant__ static const uint8_t kRhoOffsets[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                                                     25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};

struct WarpKeccak {
  uint64_t* col;        // two arrays of 5 columns x 6 words, column-major (16-byte aligned)
  uint32_t own;         // this lane's word in col
  uint32_t cm, cp;      // first words of columns x - 1 and x + 1
  uint32_t s0, s1, s2;  // pi sources of (x, y), (x + 1, y), (x + 2, y)
  uint32_t swap, rot;   // rho[x, y] as a half swap (bit 5) and a funnel shift
  uint64_t rc_mask;     // all ones on lane 0
  bool stores;

  __device__ WarpKeccak(uint32_t lane, uint64_t* smem) : col(smem) {
    const uint32_t t = lane < 25 ? lane : 0;
    const uint32_t x = t % 5, y = t / 5;
    own = 6 * x + y;
    cm = 6 * ((x + 4) % 5);
    cp = 6 * ((x + 1) % 5);
    // B[X, Y] = rotl(A'[xs, ys]) with X = ys, Y = 2 xs + 3 ys (mod 5); 2^-1 = 3 (mod 5)
    auto src = [](uint32_t X, uint32_t Y) { return (((Y + 15 - 3 * X) % 5) * 3) % 5 + 5 * X; };
    s0 = src(x, y);
    s1 = src((x + 1) % 5, y);
    s2 = src((x + 2) % 5, y);
    const uint32_t r = kRhoOffsets[t];
    swap = r & 32u;
    rot = r & 31u;
    rc_mask = lane == 0 ? ~0ull : 0ull;
    stores = lane < 25;
  }

  __device__ __forceinline__ void permute(uint64_t& a) const {
    // all 24 rounds unrolled: the round constants are immediates
#pragma unroll
    for (int r = 0; r < 24; r += 8) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        uint64_t* const c = col + 32 * (k & 1);
        if (stores) c[own] = a;
        __syncwarp();
        const ulonglong2 m01 = *reinterpret_cast<const ulonglong2*>(c + cm);
        const ulonglong2 m23 = *reinterpret_cast<const ulonglong2*>(c + cm + 2);
        const uint64_t m4 = c[cm + 4];
        const ulonglong2 p01 = *reinterpret_cast<const ulonglong2*>(c + cp);
        const ulonglong2 p23 = *reinterpret_cast<const ulonglong2*>(c + cp + 2);
        const uint64_t p4 = c[cp + 4];
        const uint64_t c_m = xor3_64(xor3_64(m01.x, m01.y, m23.x), m23.y, m4);
        const uint64_t c_p = xor3_64(xor3_64(p01.x, p01.y, p23.x), p23.y, p4);
        const uint64_t t = xor3_64(a, c_m, rotl<1>(c_p));
        const uint32_t lo = (uint32_t)t, hi = (uint32_t)(t >> 32);
        const uint32_t l2 = swap ? hi : lo, h2 = swap ? lo : hi;
        const uint64_t e = ((uint64_t)__funnelshift_l(l2, h2, rot) << 32) | __funnelshift_l(h2, l2, rot);
        const uint64_t b0 = __shfl_sync(0xffffffffu, e, s0) ^ (kKeccakRC[r + k] & rc_mask);
        const uint64_t b1 = __shfl_sync(0xffffffffu, e, s1);
        const uint64_t b2 = __shfl_sync(0xffffffffu, e, s2);
        a = chi_64(b0, b1, b2);
      }
    }
  }
};

// Byte k of the framed word-digest input: u32 len || "AppleZKProver.M31Sumcheck.Words.V1"
// || u32 1 || u64 count || words (little-endian) (SumcheckOracle.swift:1288-1299).
__device__ __forceinline__ uint32_t digest_stream_byte(const uint32_t* words, uint64_t count, uint64_t k) {
  const char dom[] = "AppleZKProver.M31Sumcheck.Words.V1";
  if (k < 4) return (34u >> (8 * k)) & 0xFFu;
  if (k < 38) return (uint8_t)dom[k - 4];
  if (k < 42) return (1u >> (8 * (k - 38))) & 0xFFu;
  if (k < 50) return (uint32_t)(count >> (8 * (k - 42))) & 0xFFu;
  const uint64_t w = (k - 50) >> 2;
  return (__ldg(words + w) >> (8 * ((k - 50) & 3))) & 0xFFu;
}

// Rate word `lane` (< 17) of the block starting at stream byte `pos` >= 136 when
// the block lies inside the stream: after the 50-byte header every 8-byte word
// starts 2 bytes into a table word, so it is assembled from three table words.
// The three words are loaded before a permutation and assembled after it, so the
// load latency hides behind the permutation instead of stalling before it.
struct BlockWords {
  uint32_t w0 = 0, w1 = 0, w2 = 0;
  __device__ __forceinline__ void load(const uint32_t* words, uint64_t pos, uint32_t lane) {
    const uint32_t* w = words + ((pos - 50) >> 2) + 2 * lane;
    w0 = __ldg(w);
    w1 = __ldg(w + 1);
    w2 = __ldg(w + 2);
  }
  __device__ __forceinline__ uint64_t word() const { return ((uint64_t)w0 >> 16) | ((uint64_t)w1 << 16) | ((uint64_t)w2 << 48); }
};

// SHA3-256 of the framed table, by the whole warp (`col`: its 64-word shared
// exchange array, 16-byte aligned); lanes 0..3 return the digest lanes.
__device__ uint64_t digest_words_warp(const uint32_t* words, uint64_t count, uint64_t* col) {
  const uint32_t lane = threadIdx.x & 31;
  const WarpKeccak kf(lane, col);
  const uint64_t total = 50 + 4 * count;
  uint64_t a = 0;
  uint64_t pos = 0;
  if (total >= 136) {
    // first block: header bytes then table bytes
    if (lane < 17) {
      uint64_t v = 0;
      for (uint32_t b = 0; b < 8; b++) v |= (uint64_t)digest_stream_byte(words, count, 8 * lane + b) << (8 * b);
      a ^= v;
    }
    pos = 136;
    // full middle blocks, the next block's words loaded before this permutation
    BlockWords next;
    if (lane < 17 && pos + 136 <= total) next.load(words, pos, lane);
    kf.permute(a);
    while (pos + 136 <= total) {
      a ^= next.word();
      const uint64_t npos = pos + 136;
      next = BlockWords();
      if (lane < 17 && npos + 136 <= total) next.load(words, npos, lane);
      kf.permute(a);
      pos = npos;
    }
  }
  // final block: tail bytes, suffix 0x06, 0x80 at the end of the rate
  const uint64_t tail = total - pos;
  if (lane < 17) {
    uint64_t v = 0;
    for (uint32_t b = 0; b < 8; b++) {
      const uint64_t k = 8 * lane + b;
      if (k < tail) v |= (uint64_t)digest_stream_byte(words, count, pos + k) << (8 * b);
      if (k == tail) v |= (uint64_t)0x06 << (8 * b);
    }
    if (lane == 16) v ^= kPadEnd;
    a ^= v;
  }
  kf.permute(a);
  return a;
}

// Even and odd sums of the 4-word groups [4j, 4j + 4) for j = t0, t0 + step, ...
// < quarter: eight 16-byte loads in flight per thread.
__device__ __forceinline__ void pair_sums(const uint4* __restrict__ q, uint64_t quarter, uint64_t t0, uint64_t step, uint32_t& z, uint32_t& o) {
  for (uint64_t j = t0; j < quarter; j += 8 * step) {
    uint4 v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      const uint64_t jj = j + k * step;
      v[k] = jj < quarter ? __ldg(q + jj) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int k = 0; k < 8; k++) {
      z = m31_add(z, m31_add(v[k].x, v[k].z));
      o = m31_add(o, m31_add(v[k].y, v[k].w));
    }
  }
}

// The threads that prove one table.  CtaGroup: a whole CTA (the single-table
// kernel).  PackedGroup: warps g, g + 4, g + 8, g + 12 of a 16-warp CTA, which
// the SM places on one sub-partition, with named barrier g + 1.
struct CtaGroup {
  __device__ uint32_t tid() const { return threadIdx.x; }
  __device__ uint32_t size() const { return blockDim.x; }
  __device__ void sync() const { __syncthreads(); }
};
constexpr uint32_t kPackedTables = 4;  // tables per packed CTA, one per sub-partition
constexpr uint32_t kPackedWarps = 4;   // warps per packed table
struct PackedGroup {
  uint32_t g;
  __device__ uint32_t tid() const { return (threadIdx.x >> 7) * 32 + (threadIdx.x & 31); }
  __device__ uint32_t size() const { return 32 * kPackedWarps; }
  __device__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(32 * kPackedWarps) : "memory"); }
};

// A group's shared scratch: the digest warp's exchange arrays, per-warp partial
// sums, the broadcast challenge and the digest.
struct SumcheckShared {
  __align__(16) uint64_t col[64];
  uint32_t red[2][32];
  uint32_t ch;
  uint64_t digest[4];
};

// Sum of v over the group, valid in the group's thread 0 (values < 2^31, reduced
// at every step).  Two arrays alternate, so one barrier per call suffices: thread
// 0 reads a call's array before it reaches the next call's barrier, which every
// writer of the call after that must pass first.
template <class G>
__device__ __forceinline__ uint32_t group_sum_m31(const G& grp, uint32_t v, uint32_t (&red)[2][32], uint32_t& parity) {
  for (int o = 16; o > 0; o >>= 1) v = m31_add(v, __shfl_down_sync(0xffffffffu, v, o));
  const uint32_t t = grp.tid();
  uint32_t* r = red[parity];
  parity ^= 1u;
  if ((t & 31) == 0) r[t >> 5] = v;
  grp.sync();
  uint32_t w = 0;
  if (t == 0)
    for (uint32_t k = 0; k < (grp.size() >> 5); k++) w = m31_add(w, r[k]);
  return w;
}

// One table on one group.  The group's first warp computes the statement's word
// digest while its other warps sum the table's even and odd entries (round 0's
// two sums; together the claimed sum), which need no challenge.  Then each round
// is a transcript round by the group's thread 0 (round frame, challenge frame,
// squeeze one word mod p) and one pass over the table that folds it,
// t'[i] = (1 - r) t[2i] + r t[2i+1], and sums the folded table's even and odd
// entries for the next round, so after the digest the table is read once per
// round.  One launch per table (or per batch of tables) leaves no launch in the
// stream waiting behind the digest, so a stream that shares a hardware work queue
// with others never holds that queue for the digest's duration.
template <class G>
__device__ void sumcheck_prove_group(const G& grp, SumcheckShared& sh, const uint32_t* __restrict__ evals, uint32_t log_n,
                                     uint32_t* __restrict__ scratch, SumcheckOut* __restrict__ out) {
  const uint64_t n = 1ull << log_n;
  const uint32_t t = grp.tid(), nt = grp.size();
  uint32_t parity = 0;
  uint32_t z = 0, o = 0;
  if (t < 32) {
    const uint64_t d = digest_words_warp(evals, n, sh.col);
    if (t < 4) sh.digest[t] = d;
  } else if (n >= 4) {
    pair_sums(reinterpret_cast<const uint4*>(evals), n >> 2, t - 32, nt - 32, z, o);
  } else if (n == 2 && t == 32) {
    z = evals[0];
    o = evals[1];
  }
  uint32_t zs = group_sum_m31(grp, z, sh.red, parity);
  uint32_t os = group_sum_m31(grp, o, sh.red, parity);
  // group_sum_m31's value is valid in thread 0, which alone runs the transcript
  // (the digest lanes are visible to it after the first sum's barrier)
  const uint32_t total = m31_add(zs, os);
  Transcript tr;
  if (t == 0) {
    out->claimed_sum = total;
    for (int i = 0; i < 4; i++) out->digest[i] = sh.digest[i];
    tr_reset(tr);
    FrameBuf f;
    sc_frame(f, 0);
    fb_u64(f, n);
    fb_u32(f, log_n);
    fb_u32(f, total);
    for (int i = 0; i < 4; i++) fb_u64(f, sh.digest[i]);
    tr_absorb(tr, f.b, f.n);
  }
  const uint32_t* cur = evals;
  uint32_t* bufs[2] = {scratch, scratch + (n >> 1)};
  // the result arrays' addresses, read once (`out` may be host memory mapped
  // into the device's address space)
  uint32_t *r0 = nullptr, *r1 = nullptr, *chs = nullptr;
  if (t == 0) {
    r0 = out->r0;
    r1 = out->r1;
    chs = out->challenges;
  }
  for (uint32_t r = 0; r < log_n; r++) {
    const uint64_t half = (n >> r) >> 1;
    if (t == 0) {
      r0[r] = zs;
      r1[r] = os;
      FrameBuf f;
      sc_frame(f, 1);
      fb_u32(f, r);
      fb_u32(f, zs);
      fb_u32(f, os);
      tr_absorb(tr, f.b, f.n);
      sc_frame(f, 2);
      fb_u32(f, r);
      fb_u32(f, kP);
      tr_absorb(tr, f.b, f.n);
      uint32_t c;
      tr_squeeze_u32(tr, 1, kP, &c);
      chs[r] = c;
      sh.ch = c;
    }
    grp.sync();
    const uint32_t c = sh.ch;
    const uint32_t omc = m31_sub(1, c);
    uint32_t* nxt = bufs[r & 1];
    z = 0;
    o = 0;
    if (half >= 2) {
      // groups of 4 entries fold into 2: 16-byte loads, 8-byte stores, 8 in flight
      const uint4* q = reinterpret_cast<const uint4*>(cur);
      uint2* w = reinterpret_cast<uint2*>(nxt);
      const uint64_t quarter = half >> 1;
      for (uint64_t j = t; j < quarter; j += 8 * (uint64_t)nt) {
        uint4 v[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const uint64_t jj = j + (uint64_t)k * nt;
          v[k] = jj < quarter ? q[jj] : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const uint64_t jj = j + (uint64_t)k * nt;
          const uint32_t e = m31_add(m31_mul(omc, v[k].x), m31_mul(c, v[k].y));
          const uint32_t d = m31_add(m31_mul(omc, v[k].z), m31_mul(c, v[k].w));
          if (jj < quarter) {
            w[jj] = make_uint2(e, d);
            z = m31_add(z, e);
            o = m31_add(o, d);
          }
        }
      }
    } else if (t == 0) {
      nxt[0] = m31_add(m31_mul(omc, cur[0]), m31_mul(c, cur[1]));
    }
    // the sums' barriers also complete nxt (and order this round's reads of sh.ch
    // before the next round's write)
    zs = group_sum_m31(grp, z, sh.red, parity);
    os = group_sum_m31(grp, o, sh.red, parity);
    cur = nxt;
  }
  if (t == 0) out->final_eval = cur[0];
}

constexpr int kSumcheckThreads = 256;
constexpr int kPackedThreads = 32 * kPackedTables * kPackedWarps;

__global__ void __launch_bounds__(kSumcheckThreads) sumcheck_kernel(const uint32_t* __restrict__ evals, uint32_t log_n, uint32_t* __restrict__ scratch,
                                                                  SumcheckOut* __restrict__ out) {
  __shared__ SumcheckShared sh;
  sumcheck_prove_group(CtaGroup{}, sh, evals, log_n, scratch, out);
}

// Up to four tables per CTA, table g on warps g, g + 4, g + 8, g + 12: the SM
// places a CTA's warps on its four sub-partitions in turn, so the four digest
// warps get a sub-partition each, beside only their own table's three summing
// warps (which wait at the first barrier once round 0's sums are done), never
// beside another of the CTA's digests.
__global__ void __launch_bounds__(kPackedThreads, 1) sumcheck_packed_kernel(const __grid_constant__ SumcheckBatch batch, uint32_t count) {
  __shared__ SumcheckShared sh[kPackedTables];
  const uint32_t g = (threadIdx.x >> 5) & (kPackedTables - 1);
  const uint32_t k = blockIdx.x * kPackedTables + g;
  if (k >= count) return;  // the group's warps all leave; no other group waits on them
  const SumcheckJob& j = batch.job[k];
  sumcheck_prove_group(PackedGroup{g}, sh[g], j.evals, j.log_n, j.scratch, j.out);
}

cudaError_t launch_sumcheck(const uint32_t* evals, uint32_t log_n, uint32_t* scratch, SumcheckOut* out, cudaStream_t s) {
  sumcheck_kernel<<<1, kSumcheckThreads, 0, s>>>(evals, log_n, scratch, out);
  return cudaGetLastError();
}

cudaError_t launch_sumcheck_batch(const SumcheckBatch& batch, uint32_t count, cudaStream_t s) {
  if (!count) return cudaSuccess;
  if (count > kSumcheckBatchMax) return cudaErrorInvalidValue;
  sumcheck_packed_kernel<<<(count + kPackedTables - 1) / kPackedTables, kPackedThreads, 0, s>>>(batch, count);
  return cudaGetLastError();
}

}  // namespace azk
