/*
 * azk_cuda.h -- C ABI of the B200 (sm_100a) commit-and-fold library.
 *
 * Drop-in boundary for AppleZKProver's Metal plans: every entry point below
 * replaces one reference API (cited as path:line inside the reference package)
 * with the same argument meaning and error behaviour.  Plain pointers and sizes
 * only; "host" pointers are CPU memory, "device" pointers come from
 * azk_buf_alloc (or any CUDA allocation on the context's device).
 *
 * Threading: every plan handle serialises its own calls with a mutex (the
 * reference's per-plan NSLock, e.g. MerkleCommitter.swift:548); distinct plans may
 * be used from different threads.  Calls are synchronous unless named _async.
 *
 * Field elements: M31 values are u32 in [0, 2^31-1); a QM31 value is four u32
 * limbs (a, b, c, d) = (a + b i) + (c + d i) u, 16 bytes little-endian.
 */
#ifndef AZK_CUDA_H
#define AZK_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes mirror AppleZKProverError (Sources/AppleZKProver/MetalTypes.swift:3-22). */
typedef enum azk_status {
  AZK_OK = 0,
  AZK_ERR_INVALID_INPUT_LAYOUT = 1,          /* .invalidInputLayout */
  AZK_ERR_INVALID_LEAF_COUNT = 2,            /* .invalidLeafCount(n) */
  AZK_ERR_UNSUPPORTED_ONE_BLOCK_LENGTH = 3,  /* .unsupportedOneBlockLength(n) */
  AZK_ERR_INVALID_PREHASHED_LEAF_LENGTH = 4, /* .invalidPrehashedLeafLength(n) */
  AZK_ERR_CORRECTNESS_VALIDATION_FAILED = 5, /* .correctnessValidationFailed(msg) */
  AZK_ERR_COMMAND_EXECUTION_FAILED = 6,      /* .commandExecutionFailed(msg) */
  AZK_ERR_UNAVAILABLE = 7,                   /* .unavailableOnThisPlatform / .noMetalDevice */
  AZK_ERR_INVALID_KERNEL_CONFIGURATION = 8,  /* .invalidKernelConfiguration(msg) */
  AZK_ERR_FAILED_TO_CREATE_BUFFER = 9,       /* .failedToCreateBuffer(label, length) */
  AZK_ERR_DEVICE_TIMEOUT = 10,               /* a bounded device wait gave up */
  AZK_ERR_HBM_BUDGET = 11                    /* admission refused: HBM budget exhausted */
} azk_status;

/* GPUExecutionStats (MetalTypes.swift:71-79): wall time of the call, device
 * time between the first and last kernel (CUDA events), host submit time. */
typedef struct azk_stats {
  double cpu_wall_s;
  double gpu_s;
  uint64_t cpu_submit_ns;
} azk_stats;

typedef struct azk_ctx azk_ctx;
typedef struct azk_keccakf_plan azk_keccakf_plan;
typedef struct azk_hash_plan azk_hash_plan;
typedef struct azk_merkle_plan azk_merkle_plan;
typedef struct azk_codeword_plan azk_codeword_plan;
typedef struct azk_pcs_prover azk_pcs_prover;
typedef struct azk_batch azk_batch;

/* ---- context and device buffers (MetalContext.swift:62-327, MetalBufferFactory.swift:8-159) ---- */

/* Create a context on CUDA device `device`.  Fails with AZK_ERR_UNAVAILABLE when
 * no sm_100 device is present (there is no CPU fallback). */
azk_status azk_ctx_create(int device, azk_ctx** out);
void azk_ctx_destroy(azk_ctx* ctx);
/* Message of the last failed call on this context (thread-local when ctx is NULL). */
const char* azk_last_error_message(const azk_ctx* ctx);
azk_status azk_ctx_device_info(azk_ctx* ctx, int* sm_count, uint64_t* total_bytes, int* cc_major, int* cc_minor);
azk_status azk_buf_alloc(azk_ctx* ctx, uint64_t bytes, void** out);
azk_status azk_buf_free(azk_ctx* ctx, void* ptr);
azk_status azk_buf_upload(azk_ctx* ctx, void* dst, uint64_t dst_offset, const void* src, uint64_t bytes);
azk_status azk_buf_download(azk_ctx* ctx, void* dst, const void* src, uint64_t src_offset, uint64_t bytes);
azk_status azk_buf_zero(azk_ctx* ctx, void* dst, uint64_t bytes);
azk_status azk_synchronize(azk_ctx* ctx);

/* ---- Keccak-f[1600] permutation batch (KeccakF1600PermutationBatcher.swift:31-70, 73-294) ----
 * Strides are multiples of 8 and >= 200; output bytes past 200 in each stride
 * are zeroed.  threads_per_block 0 selects the default. */
azk_status azk_keccakf_plan_create(azk_ctx* ctx, uint64_t count, uint64_t input_stride, uint64_t output_stride,
                                   uint32_t threads_per_block, azk_keccakf_plan** out);
azk_status azk_keccakf_plan_permute(azk_keccakf_plan* plan, const void* host_states, void* host_out, azk_stats* stats);
azk_status azk_keccakf_plan_permute_resident(azk_keccakf_plan* plan, const void* dev_in, uint64_t in_offset, void* dev_out,
                                             uint64_t out_offset, azk_stats* stats);
azk_status azk_keccakf_plan_clear(azk_keccakf_plan* plan);
void azk_keccakf_plan_destroy(azk_keccakf_plan* plan);

/* ---- fixed-rate SHA3-256 / Keccak-256 batch (SHA3BatchHasher.swift:39-264,
 * Keccak256BatchHasher.swift:5-257) ----
 * domain_suffix 0x06 = SHA3-256, 0x01 = Keccak-256.  length <= 136, stride >=
 * length, output_stride >= 32 (padding bytes zeroed). */
azk_status azk_hash_plan_create(azk_ctx* ctx, uint64_t count, uint64_t message_stride, uint64_t message_length, uint64_t output_stride,
                                uint32_t domain_suffix, uint32_t threads_per_block, azk_hash_plan** out);
azk_status azk_hash_plan_hash(azk_hash_plan* plan, const void* host_messages, void* host_digests, azk_stats* stats);
azk_status azk_hash_plan_hash_resident(azk_hash_plan* plan, const void* dev_messages, uint64_t in_offset, void* dev_digests,
                                       uint64_t out_offset, azk_stats* stats);
azk_status azk_hash_plan_clear(azk_hash_plan* plan);
void azk_hash_plan_destroy(azk_hash_plan* plan);

/* ---- SHA3 Merkle commitment over raw leaves (MerkleCommitter.swift:152-223, 526-1063) ----
 * leaf_count a power of two, leaf_length <= 136, leaf_stride >= leaf_length.
 * treelet_log: 0 = automatic, else leaves per CTA treelet = 2^treelet_log (1..13).
 * The tree stays resident after a commit, so openings gather sibling paths
 * without recomputing it. */
azk_status azk_merkle_plan_create(azk_ctx* ctx, uint64_t leaf_count, uint64_t leaf_stride, uint64_t leaf_length, uint32_t treelet_log,
                                  azk_merkle_plan** out);
azk_status azk_merkle_plan_commit(azk_merkle_plan* plan, const void* host_leaves, uint8_t root_out[32], azk_stats* stats);
azk_status azk_merkle_plan_commit_resident(azk_merkle_plan* plan, const void* dev_leaves, uint64_t offset, uint8_t root_out[32],
                                           azk_stats* stats);
/* Commit `host_leaves` and open `leaf_index`: leaf bytes, depth sibling digests
 * (bottom-up) and the root (SHA3RawLeavesMerkleCommitPlan.openRawLeaf, :667-720). */
azk_status azk_merkle_plan_open(azk_merkle_plan* plan, const void* host_leaves, uint64_t leaf_index, uint8_t* leaf_out,
                                uint8_t* siblings_out, uint8_t root_out[32], azk_stats* stats);
/* Openings of `count` leaves of the last committed tree: count * depth digests. */
azk_status azk_merkle_plan_open_resident(azk_merkle_plan* plan, const uint64_t* leaf_indices, uint64_t count, uint8_t* siblings_out,
                                         azk_stats* stats);
azk_status azk_merkle_plan_info(azk_merkle_plan* plan, uint32_t* tree_depth, uint32_t* treelet_leaf_count);
azk_status azk_merkle_plan_clear(azk_merkle_plan* plan);
void azk_merkle_plan_destroy(azk_merkle_plan* plan);
/* Root over 32-byte prehashed leaves (SHA3MerkleCommitter.commitPrehashedLeaves, :225-304;
 * SHA3PrehashedLeavesMerkleCommitPlan, :314-524). */
azk_status azk_merkle_commit_prehashed(azk_ctx* ctx, const void* host_digests, uint64_t digest_bytes, uint8_t root_out[32], azk_stats* stats);
/* SHA3PrehashedLeavesMerkleCommitPlan (MerkleCommitter.swift:314-524): the root over
 * `leaf_count` (a power of two) 32-byte digests, from host memory or resident at a
 * byte offset in device memory (commit(leafHashBuffer:leafHashOffset:), :358-398);
 * resident digests start on a 16-byte boundary. */
typedef struct azk_merkle_prehashed_plan azk_merkle_prehashed_plan;
azk_status azk_merkle_prehashed_plan_create(azk_ctx* ctx, uint64_t leaf_count, azk_merkle_prehashed_plan** out);
azk_status azk_merkle_prehashed_plan_commit(azk_merkle_prehashed_plan* plan, const void* host_digests, uint8_t root_out[32], azk_stats* stats);
azk_status azk_merkle_prehashed_plan_commit_resident(azk_merkle_prehashed_plan* plan, const void* dev_digests, uint64_t offset, uint8_t root_out[32],
                                                     azk_stats* stats);
void azk_merkle_prehashed_plan_destroy(azk_merkle_prehashed_plan* plan);

/* Merkle root of raw leaves with no device allocation: no counterpart in the
 * reference.  For callers that may not call cudaMalloc (a host that gives the
 * library a fixed memory budget, code that must not risk the implicit device
 * synchronisation of cudaMalloc/cudaFree, or a loop that cannot afford an
 * allocation failure).  All scratch lives in one fixed array inside the library's
 * device image (2 MiB + 768 bytes per device, held until the process exits); the caller
 * passes the leaves and a 32-byte root buffer on the device.  At most 65536
 * leaves (leaf_length <= 136, leaf_stride >= leaf_length); larger counts are
 * rejected with AZK_ERR_INVALID_INPUT_LAYOUT.  Work is queued on `stream`
 * (NULL = default stream) and the call returns without waiting.  The first call on
 * a device resolves the array's device address, so make it before any stream
 * capture; that address is kept for the life of the device's context, so the entry
 * point is not supported after a cudaDeviceReset in the same process.  The array is shared by every call on a device: calls whose work
 * overlaps on the GPU race and must be serialised by the caller.  Errors are
 * reported through azk_last_error_message(NULL). */
azk_status azk_merkle_root_noalloc(const void* dev_leaves, uint64_t leaf_count, uint64_t leaf_stride, uint64_t leaf_length, void* dev_root,
                                   void* stream);

/* ---- circle domain materialisation (CircleDomainMaterializationPlan.swift:52-219) ----
 * Canonical bit-reversed domain of size 2^log_size (1..26).  Points in storage
 * order as (x, y); FFT twiddles (N - 1 words, stage s at N - (N >> s)); inverse
 * domain layers for `rounds` folds concatenated (N/2 + N/4 + ... words, M31). */
azk_status azk_circle_domain_points(azk_ctx* ctx, uint32_t log_size, uint32_t* xy_out);
azk_status azk_circle_fft_twiddles(azk_ctx* ctx, uint32_t log_size, uint32_t* out);
azk_status azk_circle_inverse_layers(azk_ctx* ctx, uint32_t log_size, uint32_t rounds, uint32_t* out);
/* Plan form (CircleDomainMaterializationPlan.init, :52-133): the tables are built
 * once on the device and stay there.  At least one of points, twiddles or
 * inverse_rounds (<= log_size) is asked for.  Inverse layers are QM31 values
 * (a, 0, 0, 0), 16 bytes each, layer k (N >> (k+1) values) after layers 0..k-1. */
typedef struct azk_domain_plan azk_domain_plan;
azk_status azk_domain_plan_create(azk_ctx* ctx, uint32_t log_size, uint32_t materialize_points, uint32_t materialize_twiddles,
                                  uint32_t inverse_rounds, azk_domain_plan** out);
/* Counts (N - 1 twiddles, inverse values, values left after the rounds) and the
 * materialisation's timing (materializationStats). */
azk_status azk_domain_plan_info(azk_domain_plan* plan, uint64_t* twiddle_count, uint64_t* inverse_count, uint64_t* output_count,
                                azk_stats* materialization);
/* Device addresses of the tables, NULL for one not materialised
 * (requireDomainPointBuffer / ...TwiddleBuffer / ...InverseDomainBuffer, :135-154). */
azk_status azk_domain_plan_buffers(azk_domain_plan* plan, const void** points, const void** twiddles, const void** inverse_layers);
/* readDomainPoints (2N words, (x, y) per point in storage order), readCodewordTwiddles,
 * readInverseDomainLayers (:156-219); a table the plan did not build is
 * AZK_ERR_INVALID_INPUT_LAYOUT. */
azk_status azk_domain_plan_read_points(azk_domain_plan* plan, uint32_t* xy_out);
azk_status azk_domain_plan_read_twiddles(azk_domain_plan* plan, uint32_t* out);
azk_status azk_domain_plan_read_inverse_layers(azk_domain_plan* plan, uint32_t* out);
void azk_domain_plan_destroy(azk_domain_plan* plan);

/* ---- Circle FFT codeword (CircleCodeword.swift:411-887) ----
 * Input: N interleaved FFT-basis coefficients [x0, y0, x1, y1, ...] (QM31),
 * output: the codeword in bit-reversed domain order.  coefficient_count <= N
 * leading coefficients are given; the rest are zero. */
azk_status azk_codeword_plan_create(azk_ctx* ctx, uint32_t log_size, azk_codeword_plan** out);
azk_status azk_codeword_plan_execute(azk_codeword_plan* plan, const uint32_t* host_coefficients, uint64_t coefficient_count,
                                     uint32_t* host_codeword, azk_stats* stats);
/* Monomial polynomial P(x) + y Q(x) (CircleCodewordPlan.execute(polynomial:), :460-475). */
azk_status azk_codeword_plan_execute_polynomial(azk_codeword_plan* plan, const uint32_t* x_coefficients, uint64_t x_count,
                                                const uint32_t* y_coefficients, uint64_t y_count, uint32_t* host_codeword, azk_stats* stats);
azk_status azk_codeword_plan_execute_resident(azk_codeword_plan* plan, const void* dev_coefficients, uint64_t in_offset, void* dev_codeword,
                                              uint64_t out_offset, azk_stats* stats);
void azk_codeword_plan_destroy(azk_codeword_plan* plan);

/* ---- FRI folds (QM31FRIFold.swift:960-1877, CircleFRIFoldPlan.swift:5-518) ---- */
/* One QM31 fold with arbitrary nonzero QM31 inverse-domain points (n/2 of them). */
azk_status azk_qm31_fold(azk_ctx* ctx, const uint32_t* evaluations, uint64_t n, const uint32_t* inverse_points, const uint32_t challenge[4],
                         uint32_t* out, azk_stats* stats);
/* Circle fold chain with explicit challenges (CircleFRIFoldChainPlan, :132-280):
 * round 0 folds circle -> line, later rounds line -> line. */
azk_status azk_circle_fold_chain(azk_ctx* ctx, uint32_t log_size, const uint32_t* evaluations, const uint32_t* challenges, uint32_t rounds,
                                 uint32_t* out, azk_stats* stats);
/* QM31 fold chain, Merkle-transcript mode (QM31FRIFoldChainPlan.executeMerkleTranscriptDerived,
 * QM31FRIFold.swift:2203-2531): inverse layers are QM31 (n/2 + n/4 + ...).  Emits the
 * per-round roots (32 bytes each), challenges (4 limbs each) and the final layer. */
azk_status azk_qm31_merkle_fold_chain(azk_ctx* ctx, const uint32_t* evaluations, uint64_t n, const uint32_t* inverse_layers, uint32_t rounds,
                                      uint32_t* final_out, uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* stats);
/* QM31 fold chain challenges derived from caller-supplied commitments
 * (QM31FRIFoldTranscriptOracle.deriveChallenges, QM31FRIFold.swift:91-125). */
azk_status azk_qm31_transcript_challenges(azk_ctx* ctx, uint64_t input_count, const uint8_t* commitments, uint32_t rounds,
                                          uint32_t* challenges_out);
/* Circle Merkle-transcript fold chain with Circle V1 framing
 * (CircleFRIMerkleTranscriptFoldChainPlan, CircleFRIFoldPlan.swift:301-518). */
azk_status azk_circle_merkle_fold_chain(azk_ctx* ctx, uint32_t log_size, const uint32_t* evaluations, uint32_t log_blowup, uint32_t queries,
                                        uint32_t grinding_bits, const uint8_t public_digest[32], uint32_t rounds, uint32_t* final_out,
                                        uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* stats);
/* ---- fold plan handles ----
 * Resident entry points take (device pointer, byte offset) pairs: each range must
 * lie inside one device allocation and offsets are multiples of 16 bytes; ranges
 * the reference forbids to overlap are rejected with AZK_ERR_INVALID_INPUT_LAYOUT
 * (QM31FRIFold.swift:1236-1294, 2707-2909).  QM31 inverse-domain points are given
 * as full QM31 values (n/2 per round, concatenated round after round). */

/* QM31FRIFoldPlan (QM31FRIFold.swift:960-1338): one fold of `input_count` (even,
 * > 1) values. */
typedef struct azk_qm31_fold_plan azk_qm31_fold_plan;
azk_status azk_qm31_fold_plan_create(azk_ctx* ctx, uint64_t input_count, azk_qm31_fold_plan** out);
/* execute(evaluations:inverseDomainPoints:challenge:) (:1027-1055): host arrays. */
azk_status azk_qm31_fold_plan_execute(azk_qm31_fold_plan* plan, const uint32_t* evaluations, const uint32_t* inverse_points, const uint32_t challenge[4],
                                      uint32_t* out, azk_stats* stats);
/* executeResident (:1078-1103): the output may overlap neither input. */
azk_status azk_qm31_fold_plan_execute_resident(azk_qm31_fold_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                               const void* dev_inverse_points, uint64_t inverse_offset, void* dev_out, uint64_t out_offset,
                                               const uint32_t challenge[4], azk_stats* stats);
azk_status azk_qm31_fold_plan_clear(azk_qm31_fold_plan* plan);
void azk_qm31_fold_plan_destroy(azk_qm31_fold_plan* plan);

/* QM31FRIFoldChainPlan (QM31FRIFold.swift:1359-2931): `rounds` folds of
 * `input_count` values (every round's input count even and > 1).  The layer log
 * of the Merkle-bound mode holds each round's input layer, round r at element
 * offset n + n/2 + ... (r terms); azk_fold_chain_plan_info gives the final-layer,
 * inverse-domain and layer-log value counts. */
typedef struct azk_fold_chain_plan azk_fold_chain_plan;
azk_status azk_fold_chain_plan_create(azk_ctx* ctx, uint64_t input_count, uint32_t rounds, azk_fold_chain_plan** out);
azk_status azk_fold_chain_plan_info(azk_fold_chain_plan* plan, uint64_t* output_count, uint64_t* inverse_domain_count, uint64_t* layer_log_count);
/* Explicit challenges (execute / executeResident, :1544-1568, 1693-1721). */
azk_status azk_fold_chain_plan_execute(azk_fold_chain_plan* plan, const uint32_t* evaluations, const uint32_t* inverse_layers, const uint32_t* challenges,
                                       uint32_t* final_out, azk_stats* stats);
azk_status azk_fold_chain_plan_execute_resident(azk_fold_chain_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                                const void* dev_inverse_layers, uint64_t inverse_offset, void* dev_final, uint64_t final_offset,
                                                const uint32_t* challenges, azk_stats* stats);
/* Challenges derived from caller-given 32-byte round commitments through the QM31
 * fold transcript (executeTranscriptDerived[Resident], :1582-1614, 1723-1750);
 * resident commitments sit at `commitment_stride` (>= 32) bytes apart. */
azk_status azk_fold_chain_plan_execute_transcript(azk_fold_chain_plan* plan, const uint32_t* evaluations, const uint32_t* inverse_layers,
                                                  const uint8_t* commitments, uint32_t* final_out, uint32_t* challenges_out, azk_stats* stats);
azk_status azk_fold_chain_plan_execute_transcript_resident(azk_fold_chain_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                                           const void* dev_inverse_layers, uint64_t inverse_offset, const void* dev_commitments,
                                                           uint64_t commitments_offset, uint64_t commitment_stride, void* dev_final, uint64_t final_offset,
                                                           azk_stats* stats);
/* Merkle-bound chain: each round's layer committed (SHA3 Merkle, 16-byte QM31
 * leaves), the root absorbed and the challenge squeezed on the device; input count
 * a power of two (executeMerkleTranscriptDerived, :1637-1671). */
azk_status azk_fold_chain_plan_execute_merkle(azk_fold_chain_plan* plan, const uint32_t* evaluations, const uint32_t* inverse_layers, uint32_t* final_out,
                                              uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* stats);
/* Resident inputs, results read back (executeMerkleTranscriptDerivedReadback, :1828-1855). */
azk_status azk_fold_chain_plan_execute_merkle_readback(azk_fold_chain_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                                       const void* dev_inverse_layers, uint64_t inverse_offset, uint32_t* final_out,
                                                       uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* stats);
/* Fully resident (executeMerkleTranscriptDerivedResident, :1752-1787): commitments
 * written to dev_commitments at `commitment_stride`; dev_layer_log (may be NULL)
 * receives each round's input layer.  With dev_first_commitment (NULL for none;
 * then dev_layer_log is required) round 0's commitment is that 32-byte root instead
 * of a tree, and the layer log's first layer may be the evaluations themselves
 * (executeMerkleTranscriptDerivedResidentWithPrecomputedFirstCommitment, :1789-1826). */
azk_status azk_fold_chain_plan_execute_merkle_resident(azk_fold_chain_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                                       const void* dev_inverse_layers, uint64_t inverse_offset, void* dev_commitments,
                                                       uint64_t commitments_offset, uint64_t commitment_stride, void* dev_layer_log, uint64_t layer_log_offset,
                                                       const void* dev_first_commitment, uint64_t first_commitment_offset, void* dev_final,
                                                       uint64_t final_offset, azk_stats* stats);
/* Challenges of the plan's last execution (4 limbs per round). */
azk_status azk_fold_chain_plan_challenges(azk_fold_chain_plan* plan, uint32_t* challenges_out);
azk_status azk_fold_chain_plan_clear(azk_fold_chain_plan* plan);
void azk_fold_chain_plan_destroy(azk_fold_chain_plan* plan);

/* CircleFRIResidentQueryExtractorV1 (CircleFRIFoldPlan.swift:1027-1231): query
 * openings from committed layers already on the device (layer k of 2^(log_size-k)
 * QM31 values at element offset 2N - 2N/2^k, layers 0 .. rounds-1).  Every layer's
 * Merkle root must equal commitments[k] (else AZK_ERR_CORRECTNESS_VALIDATION_FAILED);
 * each pair index is below N/2.  Output: the queries in the proof codec's query
 * encoding (CircleProofFormat.swift:527-614), azk_query_extractor_query_bytes bytes
 * each, concatenated. */
typedef struct azk_query_extractor azk_query_extractor;
azk_status azk_query_extractor_create(azk_ctx* ctx, uint32_t log_size, uint32_t rounds, azk_query_extractor** out);
uint64_t azk_query_extractor_query_bytes(uint32_t log_size, uint32_t rounds);
azk_status azk_query_extractor_extract(azk_query_extractor* extractor, const void* dev_layers, uint64_t layers_offset, const uint8_t* commitments,
                                       const uint64_t* pair_indices, uint64_t count, uint8_t* queries_out, uint64_t* out_len, azk_stats* stats);
void azk_query_extractor_destroy(azk_query_extractor* extractor);

/* ---- Circle FRI fold plans (CircleFRIFoldPlan.swift:5-518) ----
 * The canonical domain of size 2^log_size supplies the inverse-domain layers
 * (materialised once per plan); folds run through the QM31 fold plans above, with
 * the same resident range and aliasing rules.  Evaluations are N QM31 values. */

/* CircleFRIFoldPlan (:5-130): one circle -> line fold (N -> N/2). */
typedef struct azk_circle_fold_plan azk_circle_fold_plan;
azk_status azk_circle_fold_plan_create(azk_ctx* ctx, uint32_t log_size, azk_circle_fold_plan** out);
azk_status azk_circle_fold_plan_execute(azk_circle_fold_plan* plan, const uint32_t* evaluations, const uint32_t challenge[4], uint32_t* out,
                                        azk_stats* stats);
azk_status azk_circle_fold_plan_execute_resident(azk_circle_fold_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset, void* dev_out,
                                                 uint64_t out_offset, const uint32_t challenge[4], azk_stats* stats);
/* readInverseYTwiddles (:108-110): N/2 QM31 values. */
azk_status azk_circle_fold_plan_read_inverse(azk_circle_fold_plan* plan, uint32_t* out);
azk_status azk_circle_fold_plan_clear(azk_circle_fold_plan* plan);
void azk_circle_fold_plan_destroy(azk_circle_fold_plan* plan);

/* CircleFRIFoldChainPlan (:132-280): `rounds` folds with explicit challenges
 * (round 0 circle -> line, then line -> line). */
typedef struct azk_circle_fold_chain_plan azk_circle_fold_chain_plan;
azk_status azk_circle_fold_chain_plan_create(azk_ctx* ctx, uint32_t log_size, uint32_t rounds, azk_circle_fold_chain_plan** out);
azk_status azk_circle_fold_chain_plan_execute(azk_circle_fold_chain_plan* plan, const uint32_t* evaluations, const uint32_t* challenges,
                                              uint32_t* final_out, azk_stats* stats);
azk_status azk_circle_fold_chain_plan_execute_resident(azk_circle_fold_chain_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                                       void* dev_final, uint64_t final_offset, const uint32_t* challenges, azk_stats* stats);
azk_status azk_circle_fold_chain_plan_read_inverse_layers(azk_circle_fold_chain_plan* plan, uint32_t* out);
azk_status azk_circle_fold_chain_plan_clear(azk_circle_fold_chain_plan* plan);
void azk_circle_fold_chain_plan_destroy(azk_circle_fold_chain_plan* plan);

/* CircleFRIMerkleTranscriptFoldChainPlan (:301-518): each round's layer is
 * committed as a SHA3 Merkle tree of 16-byte leaves and its challenge drawn from
 * the Circle PCS V1 transcript (header, domain, security parameters, public digest,
 * then commitment and challenge frames per round). */
typedef struct azk_circle_merkle_chain_plan azk_circle_merkle_chain_plan;
azk_status azk_circle_merkle_chain_plan_create(azk_ctx* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t queries, uint32_t grinding_bits,
                                               const uint8_t public_digest[32], uint32_t rounds, azk_circle_merkle_chain_plan** out);
/* outputCount and totalCommittedLayerCount (the committed-layer log: the input
 * layers of rounds 0..R-1, concatenated). */
azk_status azk_circle_merkle_chain_plan_info(azk_circle_merkle_chain_plan* plan, uint64_t* output_count, uint64_t* committed_layer_count);
/* execute (:391-409): final layer, 32-byte commitments and challenges read back. */
azk_status azk_circle_merkle_chain_plan_execute(azk_circle_merkle_chain_plan* plan, const uint32_t* evaluations, uint32_t* final_out,
                                                uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* stats);
/* executeResident (dev_committed_layers NULL), executeMaterializedResident
 * (committed layers written there) and ...WithPrecomputedFirstCommitment
 * (dev_first_commitment: round 0's 32-byte root, which then needs the committed
 * layer buffer) (:434-510). */
azk_status azk_circle_merkle_chain_plan_execute_resident(azk_circle_merkle_chain_plan* plan, const void* dev_evaluations, uint64_t evaluations_offset,
                                                         void* dev_committed_layers, uint64_t committed_layers_offset, void* dev_commitments,
                                                         uint64_t commitments_offset, uint64_t commitment_stride, const void* dev_first_commitment,
                                                         uint64_t first_commitment_offset, void* dev_final, uint64_t final_offset, azk_stats* stats);
/* Challenges of the last execution (4 limbs per round). */
azk_status azk_circle_merkle_chain_plan_challenges(azk_circle_merkle_chain_plan* plan, uint32_t* challenges_out);
azk_status azk_circle_merkle_chain_plan_read_inverse_layers(azk_circle_merkle_chain_plan* plan, uint32_t* out);
azk_status azk_circle_merkle_chain_plan_clear(azk_circle_merkle_chain_plan* plan);
void azk_circle_merkle_chain_plan_destroy(azk_circle_merkle_chain_plan* plan);

/* Sustained LOP3 + SHF (funnel shift) issue rate of the device, 32-bit ops per
 * second, from a probe kernel of independent chains: the integer roofline of
 * the Keccak-bound kernels (no counterpart in the reference). */
azk_status azk_probe_int_issue(azk_ctx* ctx, double* ops_per_second);
/* Canonicality gate (QM31CanonicalityCheck.swift:11-117): *non_canonical = 1 if any word >= p. */
azk_status azk_check_canonical(azk_ctx* ctx, const void* dev_words, uint64_t word_count, uint32_t* non_canonical);

/* ---- Circle PCS/FRI prover (CirclePCSFRIResidentProverV1, CircleFRIFoldPlan.swift:693-1025;
 * CircleCodewordPCSFRIProverV1, CircleCodeword.swift:920-1419) ----
 * Produces CirclePCSFRIProofCodecV1 bytes (CircleProofFormat.swift:478-593). */
typedef struct azk_schedule {
  uint32_t treelet_log;   /* leaves per CTA treelet = 2^treelet_log (1..13); 0 = default */
  uint32_t group_log;     /* upper-level group size (1..treelet_log); 0 = default */
  uint32_t threads;       /* threads per CTA for hashing kernels: 128, 256 or 512; 0 = default */
  uint32_t use_graph;     /* batched form: capture the superstep in a CUDA graph */
  /* Per-layer override: layer_treelet[L] (nonzero) is the treelet depth for a
   * committed layer of 2^L leaves; the autotuner fills this table. */
  uint8_t layer_treelet[32];
  /* Per-layer threads per CTA of the commit kernel (128, 256 or 512; 0 = `threads`)
   * for a committed layer of 2^L leaves; a launch that commits several layers takes
   * the entry of its largest one.  The autotuner fills this table too. */
  uint16_t layer_threads[32];
  /* Nonzero: each round's commit launch is a persistent grid of the resident CTAs
   * pulling treelets from a device work counter, instead of one CTA per treelet. */
  uint32_t persistent_trees;
} azk_schedule;

azk_status azk_pcs_prover_create(azk_ctx* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t queries, uint32_t grinding_bits,
                                 uint32_t rounds, const azk_schedule* schedule, azk_pcs_prover** out);
/* Bytes of the encoded proof for these parameters. */
uint64_t azk_pcs_proof_size(uint32_t log_size, uint32_t rounds, uint32_t queries, uint32_t claimed_count, uint32_t grinding_bits);
/* From codeword evaluations (bit-reversed order). */
azk_status azk_pcs_prover_prove_evaluations(azk_pcs_prover* p, const uint32_t* host_evaluations, const uint8_t public_digest[32],
                                            const uint64_t* claimed_indices, uint64_t claimed_count, uint8_t* proof_out,
                                            uint64_t* proof_len, azk_stats* stats);
/* From interleaved FFT-basis coefficients (coefficient_count leading values, rest zero):
 * FFT -> commit -> fold chain -> queries -> proof bytes, all on the device. */
azk_status azk_pcs_prover_prove_coefficients(azk_pcs_prover* p, const uint32_t* host_coefficients, uint64_t coefficient_count,
                                             const uint8_t public_digest[32], uint8_t* proof_out, uint64_t* proof_len, azk_stats* stats);
/* Resident variant: input already on the device (coefficients when
 * input_is_coefficients, else evaluations); proof bytes written to dev_proof. */
azk_status azk_pcs_prover_prove_resident(azk_pcs_prover* p, const void* dev_input, uint64_t in_offset, int input_is_coefficients,
                                         const uint8_t public_digest[32], void* dev_proof, uint64_t* proof_len, azk_stats* stats);
/* From monomial coefficient columns (x: x_count QM31, y: y_count QM31, each at most
 * N/2): converted to the FFT basis on the device by the witness kernels, then
 * proved as above (prove(polynomial:), CircleCodeword.swift:983-1005). */
azk_status azk_pcs_prover_prove_polynomial(azk_pcs_prover* p, const uint32_t* x_coefficients, uint64_t x_count, const uint32_t* y_coefficients,
                                           uint64_t y_count, const uint8_t public_digest[32], uint8_t* proof_out, uint64_t* proof_len,
                                           azk_stats* stats);
/* The same from columns resident in device memory; proof bytes written to dev_proof
 * (proveResidentCoefficients / proveResidentWitnessCoefficients, :1020-1080). */
azk_status azk_pcs_prover_prove_resident_witness(azk_pcs_prover* p, const void* dev_x, uint64_t x_offset, uint64_t x_count, const void* dev_y,
                                                 uint64_t y_offset, uint64_t y_count, const uint8_t public_digest[32], void* dev_proof,
                                                 uint64_t* proof_len, azk_stats* stats);
/* Public readbacks of the last proof: commitments (32 bytes each), challenges,
 * final layer and query pair indices (any pointer may be NULL). */
azk_status azk_pcs_prover_trace(azk_pcs_prover* p, uint8_t* commitments, uint32_t* challenges, uint32_t* final_layer, uint32_t* query_pairs);
void azk_pcs_prover_destroy(azk_pcs_prover* p);

/* ---- batched commit-and-fold superstep (no counterpart in the reference: it
 * proves one instance per plan) ----
 * Many PCS instances of uneven log sizes proved together: one launch per stage
 * over all instances (FFT passes, per-round fold + commit + transcript, queries,
 * proof emission), optionally captured in a CUDA graph. */
azk_status azk_batch_create(azk_ctx* ctx, uint32_t count, const uint32_t* log_sizes, const uint32_t* rounds, uint32_t log_blowup,
                            uint32_t queries, const azk_schedule* schedule, azk_batch** out);
/* Same with the Merkle leaf size of every committed layer: 16 bytes (one QM31
 * value per leaf, the reference's layout, CircleFRIFoldPlan.swift:1055-1062) or 64
 * bytes (four consecutive values per leaf; same transcript frames and folds, every
 * committed layer needs >= 4 values).  A 64-byte-leaf batch yields commitments,
 * challenges and final layers through azk_batch_trace; it has no proof encoding
 * (the reference's verifier opens 16-byte leaves), so azk_batch_download_proofs
 * fails and azk_batch_proof_sizes reports 0. */
azk_status azk_batch_create_leaves(azk_ctx* ctx, uint32_t count, const uint32_t* log_sizes, const uint32_t* rounds, uint32_t log_blowup,
                                   uint32_t queries, uint32_t leaf_bytes, const azk_schedule* schedule, azk_batch** out);
/* Device pointer of instance i's coefficient input (N_i QM31); the caller may
 * fill it in place (resident input).  Fetching the pointer drops what the last
 * azk_batch_upload learned about that input (its nonzero prefix, whether it is a
 * lifted M31 polynomial): fetch it again after every upload before writing
 * through it. */
azk_status azk_batch_input(azk_batch* b, uint32_t index, void** dev_input);
/* Copy coefficients from the host: instance i's coefficient_counts[i] leading
 * values start at host_coefficients + 4 * offsets[i] (u32 words / 4). */
azk_status azk_batch_upload(azk_batch* b, const uint32_t* host_coefficients, const uint64_t* offsets, const uint64_t* coefficient_counts);
/* Prove all instances from their resident coefficients.  plain != 0 runs the
 * per-instance form (each instance's kernels launched in sequence, no graph). */
azk_status azk_batch_prove(azk_batch* b, const uint8_t* public_digests, int plain, azk_stats* stats);
azk_status azk_batch_proof_sizes(azk_batch* b, uint64_t* sizes, uint64_t* total);
/* Proof bytes of all instances, concatenated in instance order. */
azk_status azk_batch_download_proofs(azk_batch* b, uint8_t* out, uint64_t capacity);
azk_status azk_batch_trace(azk_batch* b, uint32_t index, uint8_t* commitments, uint32_t* challenges, uint32_t* final_layer, uint32_t* query_pairs);
/* Per-stage CUDA-event timing of the next proves (event pairs on the batch's own
 * stream around each stage; profiled proves launch the graph's kernel sequence
 * eagerly): seconds4 = {FFT passes, per-round
 * fold+hash+transcript kernels, final folds, transcript/query/emission}. */
azk_status azk_batch_set_profiling(azk_batch* b, int enabled);
azk_status azk_batch_profile(azk_batch* b, double* seconds4);
/* Algorithmic work of one superstep: Keccak-f permutations of the tree kernels,
 * single-pass FFT bytes, final-fold bytes, and kernel launches per superstep. */
azk_status azk_batch_work(azk_batch* b, uint64_t* tree_permutations, uint64_t* fft_bytes, uint64_t* fold_bytes, uint32_t* launches);
void azk_batch_destroy(azk_batch* b);

/* ---- witness columns -> Circle FFT-basis coefficients
 * (CircleWitnessToFFTBasisPlanV1, CircleWitnessFFTBasis.swift:226-590) ----
 * For a domain of 2^log_size points (log_size 1...22): x and y monomial
 * coefficient columns (QM31, at most 2^(log_size-1) each, not both empty) become
 * the interleaved FFT-basis buffer [x0, y0, x1, y1, ...] of 2^log_size QM31 that
 * azk_pcs_prover_prove_coefficients / azk_codeword_plan_execute take.  Work grows
 * with the square of the longer column (the reference's dense matrix), without a
 * matrix in memory.  Non-canonical coefficients fail with
 * AZK_ERR_INVALID_INPUT_LAYOUT; so does a resident output that overlaps a column. */
typedef struct azk_witness_plan azk_witness_plan;
azk_status azk_witness_plan_create(azk_ctx* ctx, uint32_t log_size, azk_witness_plan** out);
azk_status azk_witness_plan_execute(azk_witness_plan* plan, const uint32_t* x_coefficients, uint64_t x_count, const uint32_t* y_coefficients,
                                    uint64_t y_count, uint32_t* fft_basis_out, azk_stats* stats);
azk_status azk_witness_plan_execute_resident(azk_witness_plan* plan, const void* dev_x, uint64_t x_offset, uint64_t x_count, const void* dev_y,
                                             uint64_t y_offset, uint64_t y_count, void* dev_out, uint64_t out_offset, azk_stats* stats);
void azk_witness_plan_destroy(azk_witness_plan* plan);

/* ---- M31 multilinear sum-check (M31MultilinearSumcheckProofBuilderV1.prove,
 * SumcheckOracle.swift:797-868) ----
 * `count` (a power of two > 1) canonical M31 evaluations; writes the per-round
 * sums over the even (sums0) and odd (sums1) entries, the transcript challenges
 * (log2(count) each), the claimed sum, the final folded evaluation and the
 * statement's word digest (SHA3-256 of the framed evaluations). */
azk_status azk_sumcheck_prove(azk_ctx* ctx, const uint32_t* evaluations, uint64_t count, uint32_t* sums0, uint32_t* sums1, uint32_t* challenges,
                              uint32_t* claimed_sum, uint32_t* final_evaluation, uint8_t digest[32], azk_stats* stats);

/* ---- continuous-batching server (no counterpart in the reference) ----
 * Jobs enter one FIFO queue; `slots` workers, each with its own CUDA stream, take
 * the front job as soon as its device memory fits `hbm_budget_bytes`, so jobs that
 * arrive while others run are admitted as slots and memory free up and their
 * kernels overlap on the device.  A worker takes a PCS job together with the other
 * queued PCS jobs of its shape (up to 8 below 2^18 values, fewer above) and proves
 * them as one batched superstep; sum-check jobs go to a lane that proves the
 * waiting tables in batched launches on its own streams.  A job larger than the
 * whole budget is refused with AZK_ERR_HBM_BUDGET at submission.  Results equal
 * those of the single-job entry points (the same kernels; only their grouping and
 * overlap differ). */
typedef struct azk_server azk_server;
azk_status azk_server_create(azk_ctx* ctx, uint64_t hbm_budget_bytes, uint32_t slots, const azk_schedule* schedule, azk_server** out);
/* Before serving: every worker proves, once, a group of zero jobs of each group size
 * of each listed shape (PCS proofs of 2^pcs_logn[i] coefficients folded for
 * pcs_rounds[i] rounds; sum-checks over 2^sumcheck_logn[i] evaluations), so its
 * device memory for those shapes, its pinned staging, its captured graphs and every
 * lazily built table exist before the first real job:
 * creating them in the middle of serving costs allocations and frees that wait for
 * the whole device.  Shapes that do not fit the HBM budget are skipped.  Returns
 * when all workers are done; warm-up jobs produce no results. */
azk_status azk_server_warm(azk_server* sv, const uint32_t* pcs_logn, const uint32_t* pcs_rounds, uint32_t n_pcs, uint32_t log_blowup,
                           uint32_t queries, const uint32_t* sumcheck_logn, uint32_t n_sumcheck);
/* Circle PCS proof from `count` leading FFT-basis coefficients (rest zero). */
azk_status azk_server_submit_pcs(azk_server* sv, uint32_t log_size, uint32_t log_blowup, uint32_t queries, uint32_t rounds, const uint32_t* coefficients,
                                 uint64_t count, const uint8_t public_digest[32], uint64_t* job_id);
/* M31 multilinear sum-check over `count` (power of two) evaluations
 * (M31MultilinearSumcheckProofBuilderV1, SumcheckOracle.swift:797-868). */
azk_status azk_server_submit_sumcheck(azk_server* sv, const uint32_t* evaluations, uint64_t count, uint64_t* job_id);
/* The same two submissions without copying the input: the server keeps the
 * address and reads the words when a worker takes the job, so they must stay
 * valid and unchanged until azk_server_poll reports the job done or failed.  The
 * arguments and the words' canonicality are checked here, as above.  Saves the
 * copy into fresh host memory (page faults included: about 1.3 ms per 4 MiB table
 * on the submitting thread). */
azk_status azk_server_submit_pcs_nocopy(azk_server* sv, uint32_t log_size, uint32_t log_blowup, uint32_t queries, uint32_t rounds,
                                        const uint32_t* coefficients, uint64_t count, const uint8_t public_digest[32], uint64_t* job_id);
azk_status azk_server_submit_sumcheck_nocopy(azk_server* sv, const uint32_t* evaluations, uint64_t count, uint64_t* job_id);
/* state: 0 queued, 1 running, 2 done, 3 failed.  Done: latency = completion -
 * submission; result = proof bytes (PCS) or u32 words {claimed sum, final
 * evaluation, digest[8], sums at 0 [rounds], sums at 1 [rounds], challenges [rounds]}
 * (sum-check); pass out = NULL to learn *out_len. */
azk_status azk_server_poll(azk_server* sv, uint64_t job_id, int* state, double* latency_s, uint8_t* out, uint64_t* out_len);
azk_status azk_server_release(azk_server* sv, uint64_t job_id);
azk_status azk_server_wait_all(azk_server* sv);
azk_status azk_server_stats(azk_server* sv, uint64_t* completed, uint64_t* elems, double* span_s, uint64_t* reserved_bytes);
/* PCS groups proved so far and the jobs they held (jobs / groups = mean group size). */
azk_status azk_server_group_stats(azk_server* sv, uint64_t* groups, uint64_t* grouped_jobs);
void azk_server_destroy(azk_server* sv);

/* ---- autotuner and learned cost model (the reference's planner races a few
 * Merkle schedules, Planner/MetalProofPlanner.swift:20-615; this replaces it) ---- */

/* Median device time of one commit-kernel launch over `concurrent` independent
 * trees of 2^log_leaves leaves: leaf_bytes 16 (QM31 leaves; fold != 0 computes
 * each leaf as a fold of a previous layer first) or 64 (raw 64-byte leaves). */
azk_status azk_tuner_time_tree(azk_ctx* ctx, uint32_t log_leaves, uint32_t leaf_bytes, uint32_t fold, uint32_t concurrent, uint32_t tile_log,
                               uint32_t group_log, uint32_t threads, uint32_t reps, double* seconds);

/* One schedule of the commit kernel, and what a race measured for it. */
typedef struct azk_tuner_candidate {
  uint32_t tile_log, group_log, threads, reserved;
} azk_tuner_candidate;
typedef struct azk_tuner_measurement {
  double median_gpu_s, p95_gpu_s, median_submit_s;
  uint32_t passed_gate; /* 0: the candidate's roots differed from the host's; not timed */
  uint32_t runs;
} azk_tuner_measurement;
/* Correctness-gated race over candidate schedules for one tree shape
 * (MetalProofPlanner.measureMerkleCandidate, Planner/MetalProofPlanner.swift:367-418):
 * a seeded random input is committed by every candidate and its roots compared with
 * the host's (the library's own host Keccak); passing candidates run warmup_runs +
 * measured_runs more times, each checked, and *winner is the one with the lowest
 * median device time plus median submit time.  Fails with
 * AZK_ERR_CORRECTNESS_VALIDATION_FAILED if no candidate passes. */
azk_status azk_tuner_race_tree(azk_ctx* ctx, uint32_t log_leaves, uint32_t leaf_bytes, uint32_t fold, uint32_t concurrent,
                               const azk_tuner_candidate* candidates, uint32_t count, uint32_t warmup_runs, uint32_t measured_runs, uint64_t seed,
                               azk_tuner_measurement* out, uint32_t* winner);
/* Randomized validation of a winner before it is persisted
 * (validateMerkleWinnerForPersistence, :447-484): `batches` fresh seeded inputs, each
 * committed and compared with the host's roots. */
azk_status azk_tuner_validate_tree(azk_ctx* ctx, uint32_t log_leaves, uint32_t leaf_bytes, uint32_t fold, uint32_t concurrent,
                                   const azk_tuner_candidate* winner, uint32_t batches, uint64_t seed);

typedef struct azk_mlp azk_mlp;
/* Fully connected network dims[0] -> ... -> dims[n_layers] (= 1), ReLU hidden
 * layers, fp32, trained on the device by hand-written forward/backward/Adam kernels. */
azk_status azk_mlp_create(azk_ctx* ctx, uint32_t n_layers, const uint32_t* dims, uint64_t seed, azk_mlp** out);
uint64_t azk_mlp_param_count(azk_mlp* mlp);
/* Parameters: per layer, weights [out][in] then biases [out]. */
azk_status azk_mlp_get_params(azk_mlp* mlp, float* params, uint64_t count);
azk_status azk_mlp_set_params(azk_mlp* mlp, const float* params, uint64_t count);
azk_status azk_mlp_forward(azk_mlp* mlp, const float* x, uint64_t rows, float* y);
/* Mean-squared-error loss and its gradient with respect to every parameter. */
azk_status azk_mlp_gradients(azk_mlp* mlp, const float* x, const float* y, uint64_t rows, float* loss, float* grads);
/* `steps` full-batch Adam steps (lr, betas 0.9/0.999); returns the final loss. */
azk_status azk_mlp_train(azk_mlp* mlp, const float* x, const float* y, uint64_t rows, uint32_t steps, float lr, float* final_loss);
void azk_mlp_destroy(azk_mlp* mlp);

#ifdef __cplusplus
}
#endif
#endif /* AZK_CUDA_H */
