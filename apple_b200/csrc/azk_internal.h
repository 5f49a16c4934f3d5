// Internal declarations shared by the kernel translation units and the C-ABI
// layer.  Nothing here is exported; include/azk_cuda.h is the public boundary.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "azk_transcript.cuh"

namespace azk {

// ---------------------------------------------------------------------------
// Merkle tree jobs.  A job commits one power-of-two tree; a launch processes a
// work list of (job, tile) pairs.  Each CTA hashes one tile of 2^tile_log leaves,
// reduces it to a treelet root in shared memory, and the last CTA to finish a
// group of 2^group_log sibling treelets (per-group arrival counter, no waiting)
// carries on with the next levels, up to the root.
// ---------------------------------------------------------------------------
enum LeafKind : uint32_t {
  kLeafRaw = 0,     // raw bytes, length <= 136, arbitrary stride
  kLeafQM31 = 1,    // 16-byte little-endian QM31 values
  kLeafFold = 2,    // fold of a previous QM31 layer, then hashed (layer written out)
  kLeafDigest = 3,  // prehashed 32-byte digests
  kLeafQM31x4 = 4,  // 64-byte leaves of 4 consecutive QM31 values
  kLeafFoldx4 = 5,  // fold of a previous layer into 4 values per 64-byte leaf, then hashed
};

enum RootAction : uint32_t {
  kRootNone = 0,
  kRootCircleRound = 1,  // Circle FRI PCS V1 transcript round -> challenge
  kRootQM31Round = 2,    // QM31 fold-chain transcript round -> challenge
};

struct TreeJob {
  uint32_t logn;       // log2(leaf count)
  uint32_t kind;       // LeafKind
  uint32_t tile_log;   // treelet depth for this job (<= logn)
  uint32_t group_log;  // levels per upper group (>= 1)
  // leaves
  const uint8_t* raw;  // kLeafRaw bytes / kLeafDigest digests
  uint64_t stride;     // kLeafRaw byte stride
  uint32_t len;        // kLeafRaw length (<= 136)
  uint32_t suffix;     // 0x06 (SHA3) or 0x01 (Keccak)
  uint32_t aligned8;   // raw base and stride are multiples of 8
  uint32_t pad0;
  const uint4* layer;  // kLeafQM31 values / kLeafFold previous layer (2n values)
  const uint32_t* inv;     // kLeafFold inverse-domain values (n)
  const uint32_t* fold_ch; // kLeafFold challenge (4 limbs)
  uint4* out_layer;        // kLeafFold output layer (n values)
  // tree storage
  uint64_t* leaf_digests;  // optional level 0 (n digests, 4 lanes each)
  uint64_t* inner;         // levels >= 1 (n - 1 digests)
  uint32_t* counters;      // zero-initialised arrival counters (self-resetting)
  // root action
  uint32_t root_action;
  uint32_t round;
  uint64_t frame_in_count;  // kRootQM31Round: layer size in the frame
  Transcript* transcript;
  uint32_t* challenge_out;  // 4 limbs
  uint64_t* root_out;       // 4 lanes
};

// Number of counters a job needs (upper bound).
inline uint64_t tree_counter_count(uint32_t logn, uint32_t tile_log) {
  uint64_t tiles = 1ull << (logn > tile_log ? logn - tile_log : 0);
  return tiles + 64;
}
// Offset (in digests) of level l >= 1 inside `inner`.
__host__ __device__ inline uint64_t inner_offset(uint32_t logn, uint32_t level) {
  uint64_t n = 1ull << logn;
  return n - ((2 * n) >> level);
}

// ---------------------------------------------------------------------------
// FFT / fold jobs
// ---------------------------------------------------------------------------
// What the upload learned about one coefficient buffer (written on the device by
// the input scan): `m31` = every coefficient below `count` has zero b, c, d limbs
// (an M31 polynomial lifted to QM31); coefficients at index >= count are zero.
// count == 0 means unknown (all N coefficients are read).
struct InputInfo {
  uint32_t m31;
  uint32_t reserved;
  uint64_t count;
};

struct FftJob {
  uint32_t logn;
  uint32_t pass;             // this job's pass index (0 reads `in`; the last pass is the low stages)
  const uint4* in;           // FFT-basis coefficients (read by the first pass)
  uint4* out;                // codeword (bit-reversed order)
  const uint32_t* tw;        // stage twiddles of the domain (N - 1 values; tw + N: the same doubled)
  uint32_t* narrow;          // N words of scratch between passes of the one-limb kernel
  const InputInfo* info;     // nonzero prefix of the input (null: all N coefficients read)
};

// Circle FFT pass geometry: the stages above bit 12 run first in chunks of at
// most 10 (strided tiles of 2^m rows x 2^c columns, c = 12 - m up to 8, so that a
// tile holds 4096 values whatever m is and a block's threads all have work), then
// one pass runs stages min(logn,12)-1 ... 0 on contiguous 4096-element tiles.
// The tile loops step one row per THREADS >> c threads, so 2^c stays <= 256, the
// smaller of the two kernels' block sizes.
static constexpr uint32_t kFftLowBits = 12;
static constexpr uint32_t kFftChunk = 10;
static constexpr uint32_t kFftMaxColsLog = 8;
struct FftPassGeom {
  uint32_t s_lo, m, c;
};
__host__ __device__ inline uint32_t fft_high_chunks(uint32_t logn) {
  return logn > kFftLowBits ? (logn - kFftLowBits + kFftChunk - 1) / kFftChunk : 0;
}
__host__ __device__ inline FftPassGeom fft_pass_geom(uint32_t logn, uint32_t pass) {
  uint32_t hc = fft_high_chunks(logn);
  if (pass < hc) {
    uint32_t top = logn - 1 - pass * kFftChunk;
    uint32_t lo = top + 1 >= kFftLowBits + kFftChunk ? top + 1 - kFftChunk : kFftLowBits;
    const uint32_t m = top - lo + 1;
    const uint32_t c = kFftLowBits - m < kFftMaxColsLog ? kFftLowBits - m : kFftMaxColsLog;
    return {lo, m, c};
  }
  uint32_t m = logn < kFftLowBits ? logn : kFftLowBits;
  return {0, m, 0};
}
__host__ __device__ inline uint64_t fft_pass_tiles(uint32_t logn, uint32_t pass) {
  FftPassGeom g = fft_pass_geom(logn, pass);
  return 1ull << (logn - g.m - g.c);
}
static constexpr uint32_t kFoldChunk = 2048;

struct FoldJob {
  uint64_t n_out;
  const uint4* prev;
  const uint32_t* inv;
  const uint32_t* ch;  // 4 limbs (device)
  uint4* out;
};

// ---------------------------------------------------------------------------
// Circle PCS prover instance (device-visible)
// ---------------------------------------------------------------------------
struct PcsInstance {
  uint32_t logn, rounds, queries, log_blowup;
  uint32_t grinding_bits, n_claimed, has_nonce, pad;
  uint64_t pub[4];
  uint64_t nonce;
  uint4* layers;          // layer k at layer_offset(k)
  uint64_t* trees;        // inner nodes of tree k at tree_offset(k)
  const uint32_t* tw;
  const uint32_t* inv;
  Transcript* transcript;
  uint32_t* challenges;   // 4 * rounds
  uint64_t* commitments;  // 4 * rounds
  uint32_t* query_pairs;  // queries
  const uint64_t* claimed;  // claimed storage indices (sorted), n_claimed
  uint8_t* proof;         // encoded proof bytes
  uint64_t proof_len;
};

__host__ __device__ inline uint64_t layer_offset(uint32_t logn, uint32_t k) {
  uint64_t n = 1ull << logn;
  return 2 * n - ((2 * n) >> k);
}
// inner nodes of tree k (levels >= 1): n_k - 1 digests
__host__ __device__ inline uint64_t tree_offset(uint32_t logn, uint32_t k) {
  uint64_t n = 1ull << logn;
  return (2 * n - ((2 * n) >> k)) - k;
}
__host__ __device__ inline uint64_t opening_bytes(uint32_t depth) { return 8 + 16 + 4 + 32ull * depth; }
__host__ __device__ inline uint64_t proof_header_bytes(uint32_t rounds, uint64_t final_count) {
  return 8 + 4 + 4 + 4 + 44 + 16 + 4 + 32 + 4 + 32ull * rounds + 8 + 16 * final_count + 4;
}
__host__ __device__ inline uint64_t proof_query_bytes(uint32_t logn, uint32_t rounds) {
  uint64_t b = 8 + 4;
  for (uint32_t k = 0; k < rounds; k++) b += 4 + 8 + 2 * opening_bytes(logn - k);
  return b;
}
__host__ __device__ inline uint64_t proof_total_bytes(uint32_t logn, uint32_t rounds, uint32_t queries, uint32_t n_claimed, bool nonce) {
  uint64_t b = proof_header_bytes(rounds, 1ull << (logn - rounds)) + (uint64_t)queries * proof_query_bytes(logn, rounds);
  if (n_claimed || nonce) b += 4 + (uint64_t)n_claimed * opening_bytes(logn);
  if (nonce) b += 8;
  return b;
}

// ---------------------------------------------------------------------------
// Launchers (defined in the .cu files)
// ---------------------------------------------------------------------------
struct LaunchCfg {
  uint32_t threads = 256;  // threads per CTA
  uint32_t grid_cap = 0;   // 0: one CTA per work item
};

cudaError_t launch_int_issue_probe(int sm_count, cudaStream_t s, uint32_t* d_sink, double* ops_per_launch, uint32_t* blocks_out);
cudaError_t prepare_tree_kernels();
cudaError_t launch_tree_direct_raw(const TreeJob& job, cudaStream_t s);
cudaError_t prepare_fft_kernels();
cudaError_t launch_keccak_permute(const uint8_t* in, uint64_t in_stride, uint8_t* out, uint64_t out_stride, uint64_t count,
                                  uint32_t threads, cudaStream_t s);
cudaError_t launch_hash_batch(const uint8_t* in, uint64_t stride, uint32_t len, uint32_t suffix, uint8_t* out, uint64_t out_stride,
                              uint64_t count, uint32_t threads, cudaStream_t s);
// `d_queue` (two zeroed words, or null): launch the persistent form, whose resident
// CTAs pull work items from that counter; null: one CTA per work item.
cudaError_t launch_tree_jobs(const TreeJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t max_tile_log, uint32_t raw_kind,
                             uint32_t threads, cudaStream_t s, uint32_t* d_queue = nullptr);
cudaError_t launch_gather_openings(const TreeJob* d_job, const uint64_t* d_idx, uint32_t nidx, uint64_t* d_out, cudaStream_t s);
cudaError_t launch_domain_tables(uint32_t logn, uint32_t* d_tw, uint32_t* d_inv, cudaStream_t s);
cudaError_t launch_domain_points(uint32_t logn, uint32_t* d_xy, cudaStream_t s);
cudaError_t launch_widen_m31(const uint32_t* d_in, uint4* d_out, uint64_t n, cudaStream_t s);
// Witness columns -> FFT basis (witness_kernels.cu): factorial tables of n
// entries (seg: ceil(n/1024) words of scratch), then the transform of two columns
// of count_x / count_y monomial coefficients into 2n interleaved QM31.
cudaError_t launch_witness_tables(uint64_t n, uint32_t* fact, uint32_t* seg, uint32_t* ifact, uint32_t* scale, cudaStream_t s);
cudaError_t launch_witness_transform(const uint4* x, uint64_t count_x, const uint4* y, uint64_t count_y, uint64_t n, const uint32_t* ifact,
                                     const uint32_t* scale, uint4* ax, uint4* ay, uint4* px, uint4* py, uint4* cx, uint4* cy, uint4* out,
                                     cudaStream_t s);
// QM31 values of each partial-sum buffer (px, py) the transform needs at capacity n.
uint64_t witness_partial_values(uint64_t n);

// FFT pass kernels.  kFftQM31: four-limb tiles (fft_pass_q_kernel); kFftM31Small:
// one-limb transforms below 2^12 values, one pass (fft_pass_m31_kernel);
// kFftM31Tile: one-limb passes of transforms of 2^12 or more that read the
// coefficients or an earlier pass's exchange words (fft_m31_tile_kernel);
// kFftM31Low: the low-stage last pass of one-limb transforms above 2^12, bulk-copied
// tiles in a persistent kernel (fft_m31_low_tma_kernel), which raises *status when
// a bounded wait on its copies runs out.
// kFftQ4Tile: four-limb tiles of transforms of 2^12 values or more that are not
// lifted M31 polynomials (fft_q_tile_kernel); kFftQM31 then serves the smaller ones.
enum FftKind : uint32_t { kFftQM31 = 0, kFftM31Small = 1, kFftM31Tile = 2, kFftM31Low = 3, kFftQ4Tile = 4, kFftKinds = 5 };
cudaError_t launch_fft_pass(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t kind, uint32_t* d_status, cudaStream_t s);
cudaError_t prepare_fft_m31_kernels();
cudaError_t launch_fft_m31_tiles(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s);
cudaError_t launch_fft_m31_low(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t* d_status, cudaStream_t s);
cudaError_t launch_fft_q_tiles(const FftJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s);
// Which kernel runs pass `pass` of a transform of 2^logn values, and how many
// work items (tiles) it has.
inline uint32_t fft_pass_kind(uint32_t logn, uint32_t pass, bool narrow) {
  if (!narrow) return logn < kFftLowBits ? kFftQM31 : kFftQ4Tile;
  if (logn < kFftLowBits) return kFftM31Small;
  return (pass == fft_high_chunks(logn) && pass > 0) ? kFftM31Low : kFftM31Tile;
}
inline uint64_t fft_kind_tiles(uint32_t logn, uint32_t pass, uint32_t kind) {
  return (kind == kFftM31Tile || kind == kFftM31Low || kind == kFftQ4Tile) ? (1ull << (logn - kFftLowBits)) : fft_pass_tiles(logn, pass);
}
// Canonicality gate over `count` QM31 coefficients; with `info`, also clears
// info->m31 when some coefficient has a nonzero b, c or d limb (the caller sets
// info = {1, 0, count} first).
cudaError_t launch_scan_input(const uint4* d_in, uint64_t count, uint32_t* d_bad, InputInfo* d_info, cudaStream_t s);
// The same over many coefficient buffers in one launch, which also writes zeros
// over each buffer's tail [count, n) (the coefficients past the uploaded prefix).
struct ScanJob {
  uint4* in;
  uint64_t count;
  uint64_t n;
  InputInfo* info;
};
cudaError_t launch_scan_inputs(const ScanJob* d_jobs, uint32_t njobs, uint64_t max_n, uint32_t* d_bad, cudaStream_t s);
cudaError_t launch_fold_jobs(const FoldJob* d_jobs, const uint2* d_work, uint32_t nwork, cudaStream_t s);
cudaError_t launch_fold_qm31_inv(const uint4* prev, const uint4* inv, const uint32_t* ch, uint4* out, uint64_t n_out, cudaStream_t s);
cudaError_t launch_pcs_prefix(PcsInstance* d_inst, uint32_t ninst, cudaStream_t s);
cudaError_t launch_pcs_finalize(PcsInstance* d_inst, const uint32_t* d_ids, uint32_t nids, cudaStream_t s);
cudaError_t launch_pcs_grind(PcsInstance* d_inst, uint32_t id, uint64_t start, uint64_t count, unsigned long long* d_found, cudaStream_t s);
cudaError_t launch_pcs_queries(PcsInstance* d_inst, const uint32_t* d_ids, uint32_t nids, cudaStream_t s);
cudaError_t launch_pcs_emit(PcsInstance* d_inst, const uint32_t* d_ids, uint32_t nids, uint32_t max_queries, cudaStream_t s);
// Encoded queries (proof codec layout) of one instance's resident layers and trees.
cudaError_t launch_query_extract(const PcsInstance* d_inst, const uint32_t* d_pairs, uint32_t count, uint8_t* d_out, cudaStream_t s);
cudaError_t launch_qm31_transcript_prefix(Transcript* d_t, uint64_t input_count, uint32_t rounds, cudaStream_t s);
cudaError_t launch_transcript_rounds_given(Transcript* d_t, uint32_t kind, const uint64_t* d_roots, uint32_t rounds, uint64_t input_count,
                                           uint32_t* d_ch, cudaStream_t s);
cudaError_t launch_check_canonical(const uint32_t* d_words, uint64_t nwords, uint32_t* d_flag, cudaStream_t s);

// M31 multilinear sum-check of one table per CTA (sumcheck_kernels.cu).  The kernel
// writes *out and the three per-round arrays it points to (log_n words each); all
// may be device memory or page-locked host memory.
struct SumcheckOut {
  uint32_t claimed_sum;
  uint32_t final_eval;
  uint64_t digest[4];
  uint32_t* r0;          // sums of the even entries, per round
  uint32_t* r1;          // sums of the odd entries, per round
  uint32_t* challenges;  // per round
};
struct SumcheckJob {
  const uint32_t* evals;
  uint32_t* scratch;  // 2^log_n words
  SumcheckOut* out;
  uint32_t log_n;
  uint32_t pad;
};
// Tables of one batched launch, passed by value (one CTA each).
constexpr uint32_t kSumcheckBatchMax = 32;
struct SumcheckBatch {
  SumcheckJob job[kSumcheckBatchMax];
};
cudaError_t launch_sumcheck(const uint32_t* evals, uint32_t log_n, uint32_t* scratch, SumcheckOut* out, cudaStream_t s);
cudaError_t launch_sumcheck_batch(const SumcheckBatch& batch, uint32_t count, cudaStream_t s);

}  // namespace azk
