// Plan handles for QM31 FRI folds, QM31 fold chains and resident query
// extraction -- the reference's QM31FRIFoldPlan and QM31FRIFoldChainPlan
// (QM31FRIFold.swift:960-1338, 1359-2931) and CircleFRIResidentQueryExtractorV1
// (CircleFRIFoldPlan.swift:1027-1231).
//
// Each handle owns its stream and device scratch and serialises its calls with a
// mutex.  Host entry points stage inputs in the plan's buffers and read results
// back; resident entry points take (device pointer, byte offset) pairs, check that
// every range lies inside its allocation and reject the overlaps the reference
// rejects, then run on the caller's buffers without copies.
#include <algorithm>
#include <memory>

#include "azk_field.cuh"
#include "azk_runtime.h"
#include "azk_tuned.h"

using namespace azk;

namespace {

constexpr uint64_t kQ = 16;  // bytes per QM31 value

cudaStream_t plan_stream() {
  cudaStream_t s = nullptr;
  AZK_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

void check_canonical_host(const uint32_t* v, uint64_t words) {
  layout(all_canonical(v, words), "input contains a non-canonical field element");
}
void check_nonzero_host(const uint32_t* v, uint64_t count) {
  for (uint64_t i = 0; i < count; i++) layout(v[4 * i] | v[4 * i + 1] | v[4 * i + 2] | v[4 * i + 3], "inverse-domain point is zero");
}

}  // namespace

// ---------------------------------------------------------------------------
// QM31FRIFoldPlan
// ---------------------------------------------------------------------------
struct azk_qm31_fold_plan {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint64_t n_in = 0, n_out = 0;
  DevBuf ev, inv, out, ch;
  ~azk_qm31_fold_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

static double qm31_fold_run(azk_qm31_fold_plan* p, const uint4* ev, const uint4* inv, uint4* out, const uint32_t ch[4]) {
  AZK_CU(cudaMemcpyAsync(p->ch.p, ch, 16, cudaMemcpyHostToDevice, p->s));
  GpuTimer g(p->s);
  AZK_CU(launch_fold_qm31_inv(ev, inv, p->ch.as<uint32_t>(), out, p->n_out, p->s));
  g.stop();
  return g.seconds();
}

extern "C" {

azk_status azk_qm31_fold_plan_create(azk_ctx* ctx, uint64_t input_count, azk_qm31_fold_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // QM31FRIFoldPlan.init (QM31FRIFold.swift:980-985)
    layout(input_count > 1 && input_count % 2 == 0 && input_count <= 0xFFFFFFFFull);
    AZK_CU(cudaSetDevice(ctx->device));
    auto p = std::make_unique<azk_qm31_fold_plan>();
    p->ctx = ctx;
    p->n_in = input_count;
    p->n_out = input_count / 2;
    p->s = plan_stream();
    p->ev.alloc(kQ * p->n_in, "QM31FRIFold.Evaluations");
    p->inv.alloc(kQ * p->n_out, "QM31FRIFold.InverseDomain");
    p->out.alloc(kQ * p->n_out, "QM31FRIFold.Output");
    p->ch.alloc(16, "QM31FRIFold.Challenge");
    *out = p.release();
  });
}

azk_status azk_qm31_fold_plan_execute(azk_qm31_fold_plan* p, const uint32_t* evaluations, const uint32_t* inverse_points, const uint32_t challenge[4],
                                      uint32_t* out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && evaluations && inverse_points && challenge && out);
    // validateInputs (QM31FRIFold.swift:1218-1233)
    check_canonical_host(evaluations, 4 * p->n_in);
    check_canonical_host(inverse_points, 4 * p->n_out);
    check_canonical_host(challenge, 4);
    check_nonzero_host(inverse_points, p->n_out);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->ev.p, evaluations, kQ * p->n_in, cudaMemcpyHostToDevice, p->s));
    AZK_CU(cudaMemcpyAsync(p->inv.p, inverse_points, kQ * p->n_out, cudaMemcpyHostToDevice, p->s));
    double gs = qm31_fold_run(p, p->ev.as<uint4>(), p->inv.as<uint4>(), p->out.as<uint4>(), challenge);
    AZK_CU(cudaMemcpyAsync(out, p->out.p, kQ * p->n_out, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, 0, gs);
  });
}

azk_status azk_qm31_fold_plan_execute_resident(azk_qm31_fold_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                               const void* dev_inverse_points, uint64_t inverse_offset, void* dev_out, uint64_t out_offset,
                                               const uint32_t challenge[4], azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && challenge);
    check_canonical_host(challenge, 4);
    const uint64_t in_b = kQ * p->n_in, out_b = kQ * p->n_out;
    layout(evaluations_offset % 16 == 0 && inverse_offset % 16 == 0 && out_offset % 16 == 0, "resident offsets must be multiples of 16 bytes");
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    // executeLocked's range and aliasing checks (QM31FRIFold.swift:1129-1139)
    require_device_range(dev_evaluations, evaluations_offset, in_b);
    require_device_range(dev_inverse_points, inverse_offset, out_b);
    require_device_range(dev_out, out_offset, out_b);
    layout(!ranges_overlap(dev_out, out_offset, out_b, dev_evaluations, evaluations_offset, in_b) &&
               !ranges_overlap(dev_out, out_offset, out_b, dev_inverse_points, inverse_offset, out_b),
           "the fold output overlaps an input");
    Timer t;
    auto at = [](const void* b, uint64_t o) { return reinterpret_cast<const uint4*>(static_cast<const uint8_t*>(b) + o); };
    double gs = qm31_fold_run(p, at(dev_evaluations, evaluations_offset), at(dev_inverse_points, inverse_offset),
                              reinterpret_cast<uint4*>(static_cast<uint8_t*>(dev_out) + out_offset), challenge);
    sync_stream(p->s);
    fill_stats(st, t, 0, gs);
  });
}

azk_status azk_qm31_fold_plan_clear(azk_qm31_fold_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    for (DevBuf* b : {&p->ev, &p->inv, &p->out, &p->ch}) AZK_CU(cudaMemsetAsync(b->p, 0, b->bytes, p->s));
    sync_stream(p->s);
  });
}

void azk_qm31_fold_plan_destroy(azk_qm31_fold_plan* p) { delete p; }

}  // extern "C"

// ---------------------------------------------------------------------------
// QM31FRIFoldChainPlan: `rounds` folds of an input of n values (each round's
// input count even), in three modes -- explicit challenges, challenges derived
// from caller-given round commitments (QM31 fold transcript), and Merkle-bound
// (each round's layer committed with 16-byte leaves, the root absorbed, the
// challenge squeezed; the input count a power of two).
// ---------------------------------------------------------------------------
struct azk_fold_chain_plan {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint64_t n_in = 0, n_out = 0;
  uint32_t rounds = 0;
  std::vector<uint64_t> count;    // input count of round r
  std::vector<uint64_t> offset;   // element offset of round r's layer in the layer log
  std::vector<uint64_t> inv_off;  // element offset of round r's inverse-domain layer
  uint64_t layer_log = 0, inv_total = 0;
  DevBuf ev, inv, layers, out, ch, cm, tr;
  // Merkle mode: one tree's inner nodes and counters (rounds run one after another)
  DevBuf inner, counters, jobs, work;
  std::vector<TreeJob> tree_jobs;
  std::vector<std::pair<uint64_t, uint64_t>> work_range;
  Sched sched;
  // Merkle-mode transcript: the QM31 fold chain's own frames, or (a Circle FRI
  // Merkle-transcript chain) the Circle PCS V1 frames, whose prefix comes from the
  // PCS instance fields in `pcs` (log size, security parameters, public digest)
  uint32_t root_kind = kRootQM31Round;
  DevBuf pcs;
  ~azk_fold_chain_plan() {
    if (s) cudaStreamDestroy(s);
  }
  bool merkle_capable() const { return is_pow2(n_in); }
  uint4* layer_at(uint4* base, uint32_t r) const { return base + offset[r]; }
};

namespace {

// Round r's fold from `prev` into `next` with challenge r (device limbs).
void chain_fold(azk_fold_chain_plan* p, uint32_t r, const uint4* prev, const uint4* inv, uint4* next) {
  AZK_CU(launch_fold_qm31_inv(prev, inv + p->inv_off[r], p->ch.as<uint32_t>() + 4 * r, next, p->count[r] / 2, p->s));
}

// Explicit or transcript mode (challenges already in p->ch): folds through the
// plan's layer scratch into `out`.
void chain_fold_all(azk_fold_chain_plan* p, const uint4* ev, const uint4* inv, uint4* out) {
  const uint4* prev = ev;
  for (uint32_t r = 0; r < p->rounds; r++) {
    uint4* next = r + 1 == p->rounds ? out : p->layer_at(p->layers.as<uint4>(), r + 1);
    chain_fold(p, r, prev, inv, next);
    prev = next;
  }
}

// Merkle-bound chain.  Layer r (r >= 1) is written into `log` at offset[r]; layer
// 0 is read from `ev` (copied into log[0] first when `copy_first`).  With
// `first_root` (device), round 0's commitment is that root instead of a tree.
void chain_merkle(azk_fold_chain_plan* p, const uint4* ev, const uint4* inv, uint4* log, bool copy_first, uint4* out, const uint64_t* first_root) {
  if (p->root_kind == kRootCircleRound)
    AZK_CU(launch_pcs_prefix(p->pcs.as<PcsInstance>(), 1, p->s));
  else
    AZK_CU(launch_qm31_transcript_prefix(p->tr.as<Transcript>(), p->n_in, p->rounds, p->s));
  if (copy_first) AZK_CU(cudaMemcpyAsync(log, ev, kQ * p->n_in, cudaMemcpyDeviceToDevice, p->s));
  const uint4* cur = copy_first ? log : ev;
  // per-round layer pointers in the tree jobs: rewritten for this call
  for (uint32_t r = 0; r < p->rounds; r++) p->tree_jobs[r].layer = r == 0 ? cur : p->layer_at(log, r);
  AZK_CU(cudaMemcpyAsync(p->jobs.p, p->tree_jobs.data(), sizeof(TreeJob) * p->rounds, cudaMemcpyHostToDevice, p->s));
  for (uint32_t r = 0; r < p->rounds; r++) {
    if (r == 0 && first_root) {
      AZK_CU(cudaMemcpyAsync(p->cm.p, first_root, 32, cudaMemcpyDeviceToDevice, p->s));
      AZK_CU(launch_transcript_rounds_given(p->tr.as<Transcript>(), p->root_kind, p->cm.as<uint64_t>(), 1, p->n_in, p->ch.as<uint32_t>(), p->s));
    } else {
      AZK_CU(launch_tree_jobs(p->jobs.as<TreeJob>(), p->work.as<uint2>() + p->work_range[r].first, (uint32_t)p->work_range[r].second,
                              p->tree_jobs[r].tile_log, kLeafQM31, tree_threads(p->sched, p->tree_jobs[r].logn), p->s));
    }
    uint4* next = r + 1 == p->rounds ? out : p->layer_at(log, r + 1);
    chain_fold(p, r, r == 0 ? cur : p->layer_at(log, r), inv, next);
  }
}

const uint4* dev_q(const void* b, uint64_t off) { return reinterpret_cast<const uint4*>(static_cast<const uint8_t*>(b) + off); }
uint4* dev_qw(void* b, uint64_t off) { return reinterpret_cast<uint4*>(static_cast<uint8_t*>(b) + off); }

// Host-array inputs of the chain: canonical evaluations and nonzero canonical
// inverse points (validateInputs / validateTranscriptInputs, QM31FRIFold.swift:2644-2705).
void chain_check_host(azk_fold_chain_plan* p, const uint32_t* ev, const uint32_t* inv) {
  layout(ev && inv);
  check_canonical_host(ev, 4 * p->n_in);
  check_canonical_host(inv, 4 * p->inv_total);
  check_nonzero_host(inv, p->inv_total);
}

// Resident range checks shared by every mode: evaluations, inverse layers and the
// final-layer output in range, the output overlapping neither input
// (validateNoOutputAliasing, QM31FRIFold.swift:2756-2778).
void chain_check_resident(azk_fold_chain_plan* p, const void* ev, uint64_t ev_off, const void* inv, uint64_t inv_off, const void* out, uint64_t out_off) {
  layout(ev_off % 16 == 0 && inv_off % 16 == 0 && out_off % 16 == 0, "resident offsets must be multiples of 16 bytes");
  require_device_range(ev, ev_off, kQ * p->n_in);
  require_device_range(inv, inv_off, kQ * p->inv_total);
  require_device_range(out, out_off, kQ * p->n_out);
  layout(!ranges_overlap(out, out_off, kQ * p->n_out, ev, ev_off, kQ * p->n_in) &&
             !ranges_overlap(out, out_off, kQ * p->n_out, inv, inv_off, kQ * p->inv_total),
         "the final-layer output overlaps an input");
}

// Commitment buffer of `rounds` 32-byte roots at `stride` (validateRoundCommitmentBuffer,
// QM31FRIFold.swift:2716-2738); returns its span in bytes.
uint64_t chain_check_commitments(azk_fold_chain_plan* p, const void* cm, uint64_t off, uint64_t stride) {
  layout(stride >= 32, "commitment stride must be at least 32 bytes");
  const uint64_t span = stride * (p->rounds - 1) + 32;
  require_device_range(cm, off, span);
  return span;
}

}  // namespace

extern "C" {

azk_status azk_fold_chain_plan_create(azk_ctx* ctx, uint64_t input_count, uint32_t rounds, azk_fold_chain_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // QM31FRIFoldChainPlan.init (QM31FRIFold.swift:1400-1431)
    layout(input_count > 1 && rounds > 0 && input_count <= 0xFFFFFFFFull);
    auto p = std::make_unique<azk_fold_chain_plan>();
    uint64_t c = input_count;
    for (uint32_t r = 0; r < rounds; r++) {
      layout(c > 1 && c % 2 == 0, "every round's input count must be even and greater than one");
      p->count.push_back(c);
      p->offset.push_back(p->layer_log);
      p->inv_off.push_back(p->inv_total);
      p->layer_log += c;
      p->inv_total += c / 2;
      c /= 2;
    }
    AZK_CU(cudaSetDevice(ctx->device));
    p->ctx = ctx;
    p->n_in = input_count;
    p->n_out = c;
    p->rounds = rounds;
    p->s = plan_stream();
    p->ev.alloc(kQ * p->n_in, "QM31FRIFoldChain.Evaluations");
    p->inv.alloc(kQ * p->inv_total, "QM31FRIFoldChain.InverseDomain");
    p->layers.alloc(kQ * p->layer_log, "QM31FRIFoldChain.Layers");
    p->out.alloc(kQ * p->n_out, "QM31FRIFoldChain.Output");
    p->ch.alloc(16ull * rounds, "QM31FRIFoldChain.Challenges");
    p->cm.alloc(32ull * rounds, "QM31FRIFoldChain.Commitments");
    p->tr.alloc(sizeof(Transcript), "QM31FRIFoldChain.Transcript");
    if (p->merkle_capable()) {
      // one committed tree at a time: the round-0 tree is the largest
      p->sched = resolve_schedule(nullptr, kTuned_pcs_single, kTunedThreads_pcs_single);
      const uint32_t logn = ilog2(input_count);
      std::vector<uint2> work;
      uint64_t max_counters = 0;
      for (uint32_t r = 0; r < rounds; r++) {
        const uint32_t lg = logn - r;
        TreeJob j{};
        j.logn = lg;
        j.kind = kLeafQM31;
        j.tile_log = tree_tile_log(p->sched, lg);
        j.group_log = std::max<uint32_t>(1, std::min(p->sched.group_log, j.tile_log));
        j.root_action = kRootQM31Round;
        j.round = r;
        j.frame_in_count = input_count >> r;
        j.transcript = p->tr.as<Transcript>();
        j.challenge_out = p->ch.as<uint32_t>() + 4 * r;
        j.root_out = p->cm.as<uint64_t>() + 4 * r;
        p->tree_jobs.push_back(j);
        const uint64_t tiles = 1ull << (lg - j.tile_log);
        p->work_range.push_back({work.size(), tiles});
        for (uint64_t k = 0; k < tiles; k++) work.push_back(make_uint2(r, (uint32_t)k));
        max_counters = std::max<uint64_t>(max_counters, tree_counter_count(lg, j.tile_log));
      }
      p->inner.alloc(32 * input_count, "QM31FRIFoldChain.TreeNodes");
      p->counters.alloc(4 * max_counters, "QM31FRIFoldChain.TreeCounters");
      p->jobs.alloc(sizeof(TreeJob) * rounds, "QM31FRIFoldChain.TreeJobs");
      p->work.alloc(sizeof(uint2) * work.size(), "QM31FRIFoldChain.TreeWork");
      for (auto& j : p->tree_jobs) {
        j.inner = p->inner.as<uint64_t>();
        j.counters = p->counters.as<uint32_t>();
      }
      AZK_CU(cudaMemsetAsync(p->counters.p, 0, p->counters.bytes, p->s));
      AZK_CU(cudaMemcpyAsync(p->work.p, work.data(), sizeof(uint2) * work.size(), cudaMemcpyHostToDevice, p->s));
      sync_stream(p->s);
    }
    *out = p.release();
  });
}

azk_status azk_fold_chain_plan_info(azk_fold_chain_plan* p, uint64_t* output_count, uint64_t* inverse_domain_count, uint64_t* layer_log_count) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    if (output_count) *output_count = p->n_out;
    if (inverse_domain_count) *inverse_domain_count = p->inv_total;
    if (layer_log_count) *layer_log_count = p->layer_log;
  });
}

// ---- explicit challenges (execute / executeResident, QM31FRIFold.swift:1544-1721) ----
azk_status azk_fold_chain_plan_execute(azk_fold_chain_plan* p, const uint32_t* evaluations, const uint32_t* inverse_layers, const uint32_t* challenges,
                                       uint32_t* final_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && challenges && final_out);
    chain_check_host(p, evaluations, inverse_layers);
    check_canonical_host(challenges, 4ull * p->rounds);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->ev.p, evaluations, kQ * p->n_in, cudaMemcpyHostToDevice, p->s));
    AZK_CU(cudaMemcpyAsync(p->inv.p, inverse_layers, kQ * p->inv_total, cudaMemcpyHostToDevice, p->s));
    AZK_CU(cudaMemcpyAsync(p->ch.p, challenges, 16ull * p->rounds, cudaMemcpyHostToDevice, p->s));
    GpuTimer g(p->s);
    chain_fold_all(p, p->ev.as<uint4>(), p->inv.as<uint4>(), p->out.as<uint4>());
    g.stop();
    AZK_CU(cudaMemcpyAsync(final_out, p->out.p, kQ * p->n_out, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_fold_chain_plan_execute_resident(azk_fold_chain_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                                const void* dev_inverse_layers, uint64_t inverse_offset, void* dev_final, uint64_t final_offset,
                                                const uint32_t* challenges, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && challenges);
    check_canonical_host(challenges, 4ull * p->rounds);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    chain_check_resident(p, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset, dev_final, final_offset);
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->ch.p, challenges, 16ull * p->rounds, cudaMemcpyHostToDevice, p->s));
    GpuTimer g(p->s);
    chain_fold_all(p, dev_q(dev_evaluations, evaluations_offset), dev_q(dev_inverse_layers, inverse_offset), dev_qw(dev_final, final_offset));
    g.stop();
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

// ---- challenges from given round commitments (executeTranscriptDerived[Resident],
// QM31FRIFold.swift:1582-1635, 1723-1750) ----
azk_status azk_fold_chain_plan_execute_transcript(azk_fold_chain_plan* p, const uint32_t* evaluations, const uint32_t* inverse_layers,
                                                  const uint8_t* commitments, uint32_t* final_out, uint32_t* challenges_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && commitments && final_out);
    chain_check_host(p, evaluations, inverse_layers);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->ev.p, evaluations, kQ * p->n_in, cudaMemcpyHostToDevice, p->s));
    AZK_CU(cudaMemcpyAsync(p->inv.p, inverse_layers, kQ * p->inv_total, cudaMemcpyHostToDevice, p->s));
    AZK_CU(cudaMemcpyAsync(p->cm.p, commitments, 32ull * p->rounds, cudaMemcpyHostToDevice, p->s));
    GpuTimer g(p->s);
    AZK_CU(launch_qm31_transcript_prefix(p->tr.as<Transcript>(), p->n_in, p->rounds, p->s));
    AZK_CU(launch_transcript_rounds_given(p->tr.as<Transcript>(), kRootQM31Round, p->cm.as<uint64_t>(), p->rounds, p->n_in, p->ch.as<uint32_t>(), p->s));
    chain_fold_all(p, p->ev.as<uint4>(), p->inv.as<uint4>(), p->out.as<uint4>());
    g.stop();
    AZK_CU(cudaMemcpyAsync(final_out, p->out.p, kQ * p->n_out, cudaMemcpyDeviceToHost, p->s));
    if (challenges_out) AZK_CU(cudaMemcpyAsync(challenges_out, p->ch.p, 16ull * p->rounds, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_fold_chain_plan_execute_transcript_resident(azk_fold_chain_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                                           const void* dev_inverse_layers, uint64_t inverse_offset, const void* dev_commitments,
                                                           uint64_t commitments_offset, uint64_t commitment_stride, void* dev_final, uint64_t final_offset,
                                                           azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    chain_check_resident(p, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset, dev_final, final_offset);
    const uint64_t span = chain_check_commitments(p, dev_commitments, commitments_offset, commitment_stride);
    layout(!ranges_overlap(dev_final, final_offset, kQ * p->n_out, dev_commitments, commitments_offset, span),
           "the final-layer output overlaps the commitments");
    Timer t;
    AZK_CU(cudaMemcpy2DAsync(p->cm.p, 32, static_cast<const uint8_t*>(dev_commitments) + commitments_offset, commitment_stride, 32, p->rounds,
                             cudaMemcpyDeviceToDevice, p->s));
    GpuTimer g(p->s);
    AZK_CU(launch_qm31_transcript_prefix(p->tr.as<Transcript>(), p->n_in, p->rounds, p->s));
    AZK_CU(launch_transcript_rounds_given(p->tr.as<Transcript>(), kRootQM31Round, p->cm.as<uint64_t>(), p->rounds, p->n_in, p->ch.as<uint32_t>(), p->s));
    chain_fold_all(p, dev_q(dev_evaluations, evaluations_offset), dev_q(dev_inverse_layers, inverse_offset), dev_qw(dev_final, final_offset));
    g.stop();
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

// ---- Merkle-bound chain (executeMerkleTranscriptDerived[Resident|Readback|
// ResidentWithPrecomputedFirstCommitment], QM31FRIFold.swift:1637-1855, 2203-2531) ----
azk_status azk_fold_chain_plan_execute_merkle(azk_fold_chain_plan* p, const uint32_t* evaluations, const uint32_t* inverse_layers, uint32_t* final_out,
                                              uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && final_out);
    layout(p->merkle_capable(), "the Merkle-bound chain needs a power-of-two input count");
    chain_check_host(p, evaluations, inverse_layers);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->ev.p, evaluations, kQ * p->n_in, cudaMemcpyHostToDevice, p->s));
    AZK_CU(cudaMemcpyAsync(p->inv.p, inverse_layers, kQ * p->inv_total, cudaMemcpyHostToDevice, p->s));
    GpuTimer g(p->s);
    chain_merkle(p, p->ev.as<uint4>(), p->inv.as<uint4>(), p->layers.as<uint4>(), false, p->out.as<uint4>(), nullptr);
    g.stop();
    AZK_CU(cudaMemcpyAsync(final_out, p->out.p, kQ * p->n_out, cudaMemcpyDeviceToHost, p->s));
    if (commitments_out) AZK_CU(cudaMemcpyAsync(commitments_out, p->cm.p, 32ull * p->rounds, cudaMemcpyDeviceToHost, p->s));
    if (challenges_out) AZK_CU(cudaMemcpyAsync(challenges_out, p->ch.p, 16ull * p->rounds, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_fold_chain_plan_execute_merkle_readback(azk_fold_chain_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                                       const void* dev_inverse_layers, uint64_t inverse_offset, uint32_t* final_out,
                                                       uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && final_out);
    layout(p->merkle_capable(), "the Merkle-bound chain needs a power-of-two input count");
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    chain_check_resident(p, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset, p->out.p, 0);
    Timer t;
    GpuTimer g(p->s);
    chain_merkle(p, dev_q(dev_evaluations, evaluations_offset), dev_q(dev_inverse_layers, inverse_offset), p->layers.as<uint4>(), false,
                 p->out.as<uint4>(), nullptr);
    g.stop();
    AZK_CU(cudaMemcpyAsync(final_out, p->out.p, kQ * p->n_out, cudaMemcpyDeviceToHost, p->s));
    if (commitments_out) AZK_CU(cudaMemcpyAsync(commitments_out, p->cm.p, 32ull * p->rounds, cudaMemcpyDeviceToHost, p->s));
    if (challenges_out) AZK_CU(cudaMemcpyAsync(challenges_out, p->ch.p, 16ull * p->rounds, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_fold_chain_plan_execute_merkle_resident(azk_fold_chain_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                                       const void* dev_inverse_layers, uint64_t inverse_offset, void* dev_commitments,
                                                       uint64_t commitments_offset, uint64_t commitment_stride, void* dev_layer_log, uint64_t layer_log_offset,
                                                       const void* dev_first_commitment, uint64_t first_commitment_offset, void* dev_final,
                                                       uint64_t final_offset, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    layout(p->merkle_capable(), "the Merkle-bound chain needs a power-of-two input count");
    // a precomputed first commitment is only taken with a layer log whose first
    // layer may be the evaluations themselves
    // (executeMerkleTranscriptDerivedResidentWithPrecomputedFirstCommitment, :1789-1826)
    layout(!dev_first_commitment || dev_layer_log, "a precomputed first commitment needs a layer log");
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    chain_check_resident(p, dev_evaluations, evaluations_offset, dev_inverse_layers, inverse_offset, dev_final, final_offset);
    const uint64_t cm_span = chain_check_commitments(p, dev_commitments, commitments_offset, commitment_stride);
    // validateNoCommitmentOutputAliasing (QM31FRIFold.swift:2811-2848)
    layout(!ranges_overlap(dev_commitments, commitments_offset, cm_span, dev_evaluations, evaluations_offset, kQ * p->n_in) &&
               !ranges_overlap(dev_commitments, commitments_offset, cm_span, dev_inverse_layers, inverse_offset, kQ * p->inv_total) &&
               !ranges_overlap(dev_commitments, commitments_offset, cm_span, dev_final, final_offset, kQ * p->n_out),
           "the commitment output overlaps another buffer");
    if (dev_first_commitment) require_device_range(dev_first_commitment, first_commitment_offset, 32);
    bool first_in_place = false;
    if (dev_layer_log) {
      layout(layer_log_offset % 16 == 0, "resident offsets must be multiples of 16 bytes");
      const uint64_t span = kQ * p->layer_log;
      require_device_range(dev_layer_log, layer_log_offset, span);
      // validateNoMaterializedLayerAliasing (QM31FRIFold.swift:2850-2909): the log's
      // first layer may be the evaluations only with a precomputed first commitment
      first_in_place = dev_first_commitment != nullptr &&
                       static_cast<const uint8_t*>(dev_layer_log) + layer_log_offset == static_cast<const uint8_t*>(dev_evaluations) + evaluations_offset;
      layout((first_in_place || !ranges_overlap(dev_layer_log, layer_log_offset, span, dev_evaluations, evaluations_offset, kQ * p->n_in)) &&
                 !ranges_overlap(dev_layer_log, layer_log_offset, span, dev_inverse_layers, inverse_offset, kQ * p->inv_total) &&
                 !ranges_overlap(dev_layer_log, layer_log_offset, span, dev_final, final_offset, kQ * p->n_out) &&
                 !ranges_overlap(dev_layer_log, layer_log_offset, span, dev_commitments, commitments_offset, cm_span),
             "the layer log overlaps another buffer");
    }
    Timer t;
    GpuTimer g(p->s);
    const uint64_t* first = dev_first_commitment ? reinterpret_cast<const uint64_t*>(static_cast<const uint8_t*>(dev_first_commitment) + first_commitment_offset)
                                                 : nullptr;
    if (dev_layer_log)
      chain_merkle(p, dev_q(dev_evaluations, evaluations_offset), dev_q(dev_inverse_layers, inverse_offset), dev_qw(dev_layer_log, layer_log_offset),
                   !first_in_place, dev_qw(dev_final, final_offset), first);
    else
      chain_merkle(p, dev_q(dev_evaluations, evaluations_offset), dev_q(dev_inverse_layers, inverse_offset), p->layers.as<uint4>(), false,
                   dev_qw(dev_final, final_offset), nullptr);
    AZK_CU(cudaMemcpy2DAsync(static_cast<uint8_t*>(dev_commitments) + commitments_offset, commitment_stride, p->cm.p, 32, 32, p->rounds,
                             cudaMemcpyDeviceToDevice, p->s));
    g.stop();
    sync_stream(p->s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_fold_chain_plan_challenges(azk_fold_chain_plan* p, uint32_t* challenges_out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && challenges_out);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaMemcpyAsync(challenges_out, p->ch.p, 16ull * p->rounds, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
  });
}

azk_status azk_fold_chain_plan_clear(azk_fold_chain_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    for (DevBuf* b : {&p->ev, &p->inv, &p->layers, &p->out, &p->ch, &p->cm, &p->tr})
      if (b->p) AZK_CU(cudaMemsetAsync(b->p, 0, b->bytes, p->s));
    if (p->inner.p) AZK_CU(cudaMemsetAsync(p->inner.p, 0, p->inner.bytes, p->s));
    sync_stream(p->s);
  });
}

void azk_fold_chain_plan_destroy(azk_fold_chain_plan* p) { delete p; }

}  // extern "C"

// ---------------------------------------------------------------------------
// CircleFRIResidentQueryExtractorV1: openings of query pairs from committed
// layers that are already on the device (layer k of 2^(log_size - k) QM31 values
// at element offset 2N - 2N/2^k, the layout of a proof's layer log).  The layers'
// trees are built once per call in one launch, every root is checked against the
// caller's commitment, and one block per query writes its openings in the proof
// codec's query encoding.
// ---------------------------------------------------------------------------
struct azk_query_extractor {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint32_t logn = 0, rounds = 0;
  uint64_t layer_values = 0, query_bytes = 0;
  DevBuf trees, counters, jobs, work, roots, inst, pairs, out;
  std::vector<TreeJob> tree_jobs;
  uint64_t nwork = 0;
  uint32_t max_tile = 1, threads = 256;
  ~azk_query_extractor() {
    if (s) cudaStreamDestroy(s);
  }
};

extern "C" {

azk_status azk_query_extractor_create(azk_ctx* ctx, uint32_t log_size, uint32_t rounds, azk_query_extractor** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // CircleFRIResidentQueryExtractorV1.init (CircleFRIFoldPlan.swift:1038-1063)
    layout(log_size >= 1 && log_size <= 26 && rounds >= 1 && rounds <= log_size);
    AZK_CU(cudaSetDevice(ctx->device));
    auto x = std::make_unique<azk_query_extractor>();
    x->ctx = ctx;
    x->logn = log_size;
    x->rounds = rounds;
    x->s = plan_stream();
    const uint64_t N = 1ull << log_size;
    x->layer_values = layer_offset(log_size, rounds);
    x->query_bytes = proof_query_bytes(log_size, rounds);
    Sched sc = resolve_schedule(nullptr, kTuned_pcs_single, kTunedThreads_pcs_single);
    x->threads = tree_threads(sc, log_size);  // one launch over every layer: the largest one's
    x->trees.alloc(32 * 2 * N, "QueryExtractor.Trees");
    x->roots.alloc(32ull * rounds, "QueryExtractor.Roots");
    uint64_t counters = 0;
    std::vector<uint64_t> cnt_off;
    std::vector<uint2> work;
    for (uint32_t k = 0; k < rounds; k++) {
      const uint32_t lg = log_size - k;
      TreeJob j{};
      j.logn = lg;
      j.kind = kLeafQM31;
      j.tile_log = tree_tile_log(sc, lg);
      j.group_log = std::max<uint32_t>(1, std::min(sc.group_log, j.tile_log));
      j.inner = x->trees.as<uint64_t>() + 4 * tree_offset(log_size, k);
      j.root_action = kRootNone;
      j.root_out = x->roots.as<uint64_t>() + 4 * k;
      cnt_off.push_back(counters);
      counters += tree_counter_count(lg, j.tile_log);
      x->max_tile = std::max(x->max_tile, j.tile_log);
      for (uint64_t t = 0; t < (1ull << (lg - j.tile_log)); t++) work.push_back(make_uint2(k, (uint32_t)t));
      x->tree_jobs.push_back(j);
    }
    x->counters.alloc(4 * counters, "QueryExtractor.Counters");
    for (uint32_t k = 0; k < rounds; k++) x->tree_jobs[k].counters = x->counters.as<uint32_t>() + cnt_off[k];
    x->nwork = work.size();
    x->jobs.alloc(sizeof(TreeJob) * rounds, "QueryExtractor.TreeJobs");
    x->work.alloc(sizeof(uint2) * work.size(), "QueryExtractor.TreeWork");
    x->inst.alloc(sizeof(PcsInstance), "QueryExtractor.Instance");
    AZK_CU(cudaMemsetAsync(x->counters.p, 0, x->counters.bytes, x->s));
    AZK_CU(cudaMemcpyAsync(x->work.p, work.data(), sizeof(uint2) * work.size(), cudaMemcpyHostToDevice, x->s));
    sync_stream(x->s);
    *out = x.release();
  });
}

uint64_t azk_query_extractor_query_bytes(uint32_t log_size, uint32_t rounds) {
  if (log_size < 1 || log_size > 30 || rounds < 1 || rounds > log_size) return 0;
  return proof_query_bytes(log_size, rounds);
}

azk_status azk_query_extractor_extract(azk_query_extractor* x, const void* dev_layers, uint64_t layers_offset, const uint8_t* commitments,
                                       const uint64_t* pair_indices, uint64_t count, uint8_t* queries_out, uint64_t* out_len, azk_stats* st) {
  return guarded(x ? x->ctx : nullptr, [&] {
    layout(x && commitments && pair_indices && queries_out && out_len);
    // extractQueries preconditions (CircleFRIFoldPlan.swift:1065-1095)
    layout(count >= 1 && count <= 0xFFFFFFFFull);
    const uint64_t half = 1ull << (x->logn - 1);
    std::vector<uint32_t> pairs(count);
    for (uint64_t i = 0; i < count; i++) {
      layout(pair_indices[i] < half, "query pair index out of range");
      pairs[i] = (uint32_t)pair_indices[i];
    }
    const uint64_t need = count * x->query_bytes;
    layout(*out_len >= need, "query buffer too small");
    layout(layers_offset % 16 == 0, "resident offsets must be multiples of 16 bytes");
    std::lock_guard<std::mutex> lk(x->mu);
    AZK_CU(cudaSetDevice(x->ctx->device));
    require_device_range(dev_layers, layers_offset, kQ * x->layer_values);
    Timer t;
    const uint4* layers = dev_q(dev_layers, layers_offset);
    for (uint32_t k = 0; k < x->rounds; k++) x->tree_jobs[k].layer = layers + layer_offset(x->logn, k);
    PcsInstance I{};
    I.logn = x->logn;
    I.rounds = x->rounds;
    I.layers = const_cast<uint4*>(layers);
    I.trees = x->trees.as<uint64_t>();
    if (x->pairs.bytes < 4 * count) x->pairs.alloc(4 * count, "QueryExtractor.Pairs");
    if (x->out.bytes < need) x->out.alloc(need, "QueryExtractor.Queries");
    AZK_CU(cudaMemcpyAsync(x->jobs.p, x->tree_jobs.data(), sizeof(TreeJob) * x->rounds, cudaMemcpyHostToDevice, x->s));
    AZK_CU(cudaMemcpyAsync(x->inst.p, &I, sizeof(PcsInstance), cudaMemcpyHostToDevice, x->s));
    AZK_CU(cudaMemcpyAsync(x->pairs.p, pairs.data(), 4 * count, cudaMemcpyHostToDevice, x->s));
    GpuTimer g(x->s);
    AZK_CU(launch_tree_jobs(x->jobs.as<TreeJob>(), x->work.as<uint2>(), (uint32_t)x->nwork, x->max_tile, kLeafQM31, x->threads, x->s));
    AZK_CU(launch_query_extract(x->inst.as<PcsInstance>(), x->pairs.as<uint32_t>(), (uint32_t)count, x->out.as<uint8_t>(), x->s));
    g.stop();
    std::vector<uint8_t> roots(32ull * x->rounds);
    AZK_CU(cudaMemcpyAsync(roots.data(), x->roots.p, roots.size(), cudaMemcpyDeviceToHost, x->s));
    sync_stream(x->s);
    // each layer's root must be the committed one (extractOpening, :1161-1167)
    require(std::equal(roots.begin(), roots.end(), commitments), AZK_ERR_CORRECTNESS_VALIDATION_FAILED,
            "Resident Circle FRI query opening root did not match the committed layer root.");
    AZK_CU(cudaMemcpyAsync(queries_out, x->out.p, need, cudaMemcpyDeviceToHost, x->s));
    sync_stream(x->s);
    *out_len = need;
    fill_stats(st, t, 0, g.seconds());
  });
}

void azk_query_extractor_destroy(azk_query_extractor* x) { delete x; }

}  // extern "C"

// ---------------------------------------------------------------------------
// CircleDomainMaterializationPlan (CircleDomainMaterializationPlan.swift:52-219)
// and the Circle FRI fold plans built on it (CircleFRIFoldPlan.swift:5-518): the
// canonical domain's inverse-domain layers are materialised once per plan as QM31
// values (a, 0, 0, 0) and the folds run through the QM31 fold plans above.
// ---------------------------------------------------------------------------
struct azk_domain_plan {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint32_t logn = 0, rounds = 0;
  bool points = false, twiddles = false;
  uint64_t inv_total = 0;
  DevBuf pts, tw, inv;
  double gpu_s = 0, wall_s = 0;
  ~azk_domain_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

struct azk_circle_fold_plan {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  azk_domain_plan* dom = nullptr;
  azk_qm31_fold_plan* fold = nullptr;
  ~azk_circle_fold_plan();
};

struct azk_circle_fold_chain_plan {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  azk_domain_plan* dom = nullptr;
  azk_fold_chain_plan* chain = nullptr;
  ~azk_circle_fold_chain_plan();
};

struct azk_circle_merkle_chain_plan {
  azk_ctx* ctx = nullptr;
  std::mutex mu;
  azk_domain_plan* dom = nullptr;
  azk_fold_chain_plan* chain = nullptr;
  ~azk_circle_merkle_chain_plan();
};

extern "C" {

azk_status azk_domain_plan_create(azk_ctx* ctx, uint32_t log_size, uint32_t materialize_points, uint32_t materialize_twiddles, uint32_t inverse_rounds,
                                  azk_domain_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // CircleDomainMaterializationPlan.init preconditions (:59-66)
    layout(log_size >= 1 && log_size <= 26);
    layout(materialize_points || materialize_twiddles || inverse_rounds > 0);
    layout(inverse_rounds <= log_size);
    AZK_CU(cudaSetDevice(ctx->device));
    Timer t;
    auto p = std::make_unique<azk_domain_plan>();
    p->ctx = ctx;
    p->logn = log_size;
    p->rounds = inverse_rounds;
    p->points = materialize_points != 0;
    p->twiddles = materialize_twiddles != 0;
    const uint64_t n = 1ull << log_size;
    p->inv_total = n - (n >> inverse_rounds);
    p->s = plan_stream();
    const auto& d = domain_tables(ctx, log_size);
    if (p->points) p->pts.alloc(8 * n, "CircleDomain.DomainPoints");
    if (p->twiddles) p->tw.alloc(4 * (n - 1), "CircleDomain.CodewordFFTTwiddles");
    if (inverse_rounds) p->inv.alloc(kQ * p->inv_total, "CircleDomain.InverseDomain");
    GpuTimer g(p->s);
    if (p->points) AZK_CU(launch_domain_points(log_size, p->pts.as<uint32_t>(), p->s));
    if (p->twiddles) AZK_CU(cudaMemcpyAsync(p->tw.p, d.tw, 4 * (n - 1), cudaMemcpyDeviceToDevice, p->s));
    // inverse layer k (n >> (k+1) values) sits at n - (n >> k) in the context's
    // table, the same offset the concatenated layers have here
    if (inverse_rounds) AZK_CU(launch_widen_m31(d.inv, p->inv.as<uint4>(), p->inv_total, p->s));
    g.stop();
    p->gpu_s = g.seconds();
    sync_stream(p->s);
    p->wall_s = t.seconds();
    *out = p.release();
  });
}

azk_status azk_domain_plan_info(azk_domain_plan* p, uint64_t* twiddle_count, uint64_t* inverse_count, uint64_t* output_count, azk_stats* materialization) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    const uint64_t n = 1ull << p->logn;
    if (twiddle_count) *twiddle_count = n - 1;
    if (inverse_count) *inverse_count = p->inv_total;
    if (output_count) *output_count = n >> p->rounds;
    if (materialization) {
      materialization->cpu_wall_s = p->wall_s;
      materialization->gpu_s = p->gpu_s;
      materialization->cpu_submit_ns = 0;
    }
  });
}

azk_status azk_domain_plan_buffers(azk_domain_plan* p, const void** points, const void** twiddles, const void** inverse_layers) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    if (points) *points = p->pts.p;
    if (twiddles) *twiddles = p->tw.p;
    if (inverse_layers) *inverse_layers = p->inv.p;
  });
}

static void domain_read(azk_domain_plan* p, const DevBuf& b, bool present, void* out, uint64_t bytes) {
  layout(out != nullptr);
  // requireDomainPointBuffer / requireCodewordTwiddleBuffer / requireInverseDomainBuffer (:135-154)
  require(present, AZK_ERR_INVALID_INPUT_LAYOUT, "the plan did not materialise this table");
  std::lock_guard<std::mutex> lk(p->mu);
  AZK_CU(cudaSetDevice(p->ctx->device));
  AZK_CU(cudaMemcpyAsync(out, b.p, bytes, cudaMemcpyDeviceToHost, p->s));
  sync_stream(p->s);
}

azk_status azk_domain_plan_read_points(azk_domain_plan* p, uint32_t* xy_out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    domain_read(p, p->pts, p->points, xy_out, 8ull << p->logn);
  });
}

azk_status azk_domain_plan_read_twiddles(azk_domain_plan* p, uint32_t* out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    domain_read(p, p->tw, p->twiddles, out, 4 * ((1ull << p->logn) - 1));
  });
}

azk_status azk_domain_plan_read_inverse_layers(azk_domain_plan* p, uint32_t* out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    domain_read(p, p->inv, p->rounds > 0, out, kQ * p->inv_total);
  });
}

void azk_domain_plan_destroy(azk_domain_plan* p) { delete p; }

}  // extern "C"

azk_circle_fold_plan::~azk_circle_fold_plan() {
  azk_qm31_fold_plan_destroy(fold);
  azk_domain_plan_destroy(dom);
}
azk_circle_fold_chain_plan::~azk_circle_fold_chain_plan() {
  azk_fold_chain_plan_destroy(chain);
  azk_domain_plan_destroy(dom);
}
azk_circle_merkle_chain_plan::~azk_circle_merkle_chain_plan() {
  azk_fold_chain_plan_destroy(chain);
  azk_domain_plan_destroy(dom);
}

namespace {
// A C-ABI call made inside another one: its failure becomes this call's.
void forward(azk_ctx* ctx, azk_status st) {
  if (st != AZK_OK) fail(st, azk_last_error_message(ctx));
}
}  // namespace

extern "C" {

// ---- CircleFRIFoldPlan (:5-130): circle -> line fold of the whole domain ----
azk_status azk_circle_fold_plan_create(azk_ctx* ctx, uint32_t log_size, azk_circle_fold_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && log_size >= 1 && log_size <= 26);
    auto p = std::make_unique<azk_circle_fold_plan>();
    p->ctx = ctx;
    forward(ctx, azk_domain_plan_create(ctx, log_size, 0, 0, 1, &p->dom));
    forward(ctx, azk_qm31_fold_plan_create(ctx, 1ull << log_size, &p->fold));
    *out = p.release();
  });
}

azk_status azk_circle_fold_plan_execute(azk_circle_fold_plan* p, const uint32_t* evaluations, const uint32_t challenge[4], uint32_t* out,
                                        azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && evaluations && challenge && out);
    const uint64_t n = 1ull << p->dom->logn;
    check_canonical_host(evaluations, 4 * n);
    check_canonical_host(challenge, 4);
    std::lock_guard<std::mutex> lk(p->mu);
    azk_qm31_fold_plan* f = p->fold;
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(f->ev.p, evaluations, kQ * n, cudaMemcpyHostToDevice, f->s));
    azk_stats inner{};
    forward(p->ctx, azk_qm31_fold_plan_execute_resident(f, f->ev.p, 0, p->dom->inv.p, 0, f->out.p, 0, challenge, &inner));
    AZK_CU(cudaMemcpyAsync(out, f->out.p, kQ * (n / 2), cudaMemcpyDeviceToHost, f->s));
    sync_stream(f->s);
    fill_stats(st, t, 0, inner.gpu_s);
  });
}

azk_status azk_circle_fold_plan_execute_resident(azk_circle_fold_plan* p, const void* dev_evaluations, uint64_t evaluations_offset, void* dev_out,
                                                 uint64_t out_offset, const uint32_t challenge[4], azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    forward(p->ctx, azk_qm31_fold_plan_execute_resident(p->fold, dev_evaluations, evaluations_offset, p->dom->inv.p, 0, dev_out, out_offset, challenge, st));
  });
}

azk_status azk_circle_fold_plan_read_inverse(azk_circle_fold_plan* p, uint32_t* out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_domain_plan_read_inverse_layers(p->dom, out));
  });
}

azk_status azk_circle_fold_plan_clear(azk_circle_fold_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_qm31_fold_plan_clear(p->fold));
  });
}

void azk_circle_fold_plan_destroy(azk_circle_fold_plan* p) { delete p; }

// ---- CircleFRIFoldChainPlan (:132-280): explicit challenges ----
azk_status azk_circle_fold_chain_plan_create(azk_ctx* ctx, uint32_t log_size, uint32_t rounds, azk_circle_fold_chain_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && log_size >= 1 && log_size <= 26 && rounds >= 1 && rounds <= log_size);
    auto p = std::make_unique<azk_circle_fold_chain_plan>();
    p->ctx = ctx;
    forward(ctx, azk_domain_plan_create(ctx, log_size, 0, 0, rounds, &p->dom));
    forward(ctx, azk_fold_chain_plan_create(ctx, 1ull << log_size, rounds, &p->chain));
    *out = p.release();
  });
}

azk_status azk_circle_fold_chain_plan_execute(azk_circle_fold_chain_plan* p, const uint32_t* evaluations, const uint32_t* challenges, uint32_t* final_out,
                                              azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && evaluations && challenges && final_out);
    azk_fold_chain_plan* c = p->chain;
    check_canonical_host(evaluations, 4 * c->n_in);
    check_canonical_host(challenges, 4ull * c->rounds);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(c->ev.p, evaluations, kQ * c->n_in, cudaMemcpyHostToDevice, c->s));
    azk_stats inner{};
    forward(p->ctx, azk_fold_chain_plan_execute_resident(c, c->ev.p, 0, p->dom->inv.p, 0, c->out.p, 0, challenges, &inner));
    AZK_CU(cudaMemcpyAsync(final_out, c->out.p, kQ * c->n_out, cudaMemcpyDeviceToHost, c->s));
    sync_stream(c->s);
    fill_stats(st, t, 0, inner.gpu_s);
  });
}

azk_status azk_circle_fold_chain_plan_execute_resident(azk_circle_fold_chain_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                                       void* dev_final, uint64_t final_offset, const uint32_t* challenges, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    forward(p->ctx, azk_fold_chain_plan_execute_resident(p->chain, dev_evaluations, evaluations_offset, p->dom->inv.p, 0, dev_final, final_offset,
                                                         challenges, st));
  });
}

azk_status azk_circle_fold_chain_plan_read_inverse_layers(azk_circle_fold_chain_plan* p, uint32_t* out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_domain_plan_read_inverse_layers(p->dom, out));
  });
}

azk_status azk_circle_fold_chain_plan_clear(azk_circle_fold_chain_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_fold_chain_plan_clear(p->chain));
  });
}

void azk_circle_fold_chain_plan_destroy(azk_circle_fold_chain_plan* p) { delete p; }

// ---- CircleFRIMerkleTranscriptFoldChainPlan (:301-518): Circle PCS V1 frames ----
azk_status azk_circle_merkle_chain_plan_create(azk_ctx* ctx, uint32_t log_size, uint32_t log_blowup, uint32_t queries, uint32_t grinding_bits,
                                               const uint8_t public_digest[32], uint32_t rounds, azk_circle_merkle_chain_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && public_digest);
    // init preconditions (:344-350) and CircleFRISecurityParametersV1 (CircleProofFormat.swift:136-151)
    layout(log_size >= 1 && log_size <= 26 && rounds >= 1 && rounds <= log_size);
    layout(log_blowup > 0 && queries > 0 && grinding_bits <= 20 && (uint64_t)log_blowup * queries + grinding_bits <= 0xFFFFFFFFull);
    auto p = std::make_unique<azk_circle_merkle_chain_plan>();
    p->ctx = ctx;
    forward(ctx, azk_domain_plan_create(ctx, log_size, 0, 0, rounds, &p->dom));
    forward(ctx, azk_fold_chain_plan_create(ctx, 1ull << log_size, rounds, &p->chain));
    azk_fold_chain_plan* c = p->chain;
    // the prefix frames come from a PCS instance record: log size, security
    // parameters, public digest and the transcript they are absorbed into
    PcsInstance I{};
    I.logn = log_size;
    I.rounds = rounds;
    I.queries = queries;
    I.log_blowup = log_blowup;
    I.grinding_bits = grinding_bits;
    std::memcpy(I.pub, public_digest, 32);
    I.transcript = c->tr.as<Transcript>();
    c->pcs.alloc(sizeof(PcsInstance), "CircleFRIMerkleChain.Instance");
    AZK_CU(cudaMemcpyAsync(c->pcs.p, &I, sizeof(PcsInstance), cudaMemcpyHostToDevice, c->s));
    sync_stream(c->s);
    c->root_kind = kRootCircleRound;
    for (auto& j : c->tree_jobs) j.root_action = kRootCircleRound;
    *out = p.release();
  });
}

azk_status azk_circle_merkle_chain_plan_info(azk_circle_merkle_chain_plan* p, uint64_t* output_count, uint64_t* committed_layer_count) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    if (output_count) *output_count = p->chain->n_out;
    if (committed_layer_count) *committed_layer_count = p->chain->layer_log;
  });
}

azk_status azk_circle_merkle_chain_plan_execute(azk_circle_merkle_chain_plan* p, const uint32_t* evaluations, uint32_t* final_out,
                                                uint8_t* commitments_out, uint32_t* challenges_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && evaluations && final_out);
    azk_fold_chain_plan* c = p->chain;
    check_canonical_host(evaluations, 4 * c->n_in);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(c->ev.p, evaluations, kQ * c->n_in, cudaMemcpyHostToDevice, c->s));
    azk_stats inner{};
    forward(p->ctx, azk_fold_chain_plan_execute_merkle_readback(c, c->ev.p, 0, p->dom->inv.p, 0, final_out, commitments_out, challenges_out, &inner));
    fill_stats(st, t, 0, inner.gpu_s);
  });
}

azk_status azk_circle_merkle_chain_plan_execute_resident(azk_circle_merkle_chain_plan* p, const void* dev_evaluations, uint64_t evaluations_offset,
                                                         void* dev_committed_layers, uint64_t committed_layers_offset, void* dev_commitments,
                                                         uint64_t commitments_offset, uint64_t commitment_stride, const void* dev_first_commitment,
                                                         uint64_t first_commitment_offset, void* dev_final, uint64_t final_offset, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    forward(p->ctx, azk_fold_chain_plan_execute_merkle_resident(p->chain, dev_evaluations, evaluations_offset, p->dom->inv.p, 0, dev_commitments,
                                                                commitments_offset, commitment_stride, dev_committed_layers, committed_layers_offset,
                                                                dev_first_commitment, first_commitment_offset, dev_final, final_offset, st));
  });
}

azk_status azk_circle_merkle_chain_plan_challenges(azk_circle_merkle_chain_plan* p, uint32_t* challenges_out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_fold_chain_plan_challenges(p->chain, challenges_out));
  });
}

azk_status azk_circle_merkle_chain_plan_read_inverse_layers(azk_circle_merkle_chain_plan* p, uint32_t* out) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_domain_plan_read_inverse_layers(p->dom, out));
  });
}

azk_status azk_circle_merkle_chain_plan_clear(azk_circle_merkle_chain_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    forward(p->ctx, azk_fold_chain_plan_clear(p->chain));
  });
}

void azk_circle_merkle_chain_plan_destroy(azk_circle_merkle_chain_plan* p) { delete p; }

}  // extern "C"
