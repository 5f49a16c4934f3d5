// Circle PCS/FRI proving engine: FFT -> per-round (fold + leaf hash + treelet +
// upper tree + transcript) -> final fold -> final-layer binding -> queries ->
// proof bytes, for one instance (azk_pcs_prover, mirroring
// CirclePCSFRIResidentProverV1 / CircleCodewordPCSFRIProverV1) or many uneven
// instances at once (azk_batch).
//
// Batched form: each stage is one launch over the work items of every instance
// still active in that round, so small instances share the GPU with large ones
// and the whole superstep is a fixed launch sequence captured in a CUDA graph.
// Plain form: the same kernels, launched instance after instance.
#include <memory>
#include <algorithm>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

#include "azk_field.cuh"
#include "azk_runtime.h"
#include "azk_tuned.h"

namespace azk {
struct SumcheckOut {
  uint32_t claimed_sum;
  uint32_t final_eval;
  uint64_t digest[4];
  uint32_t* r0;
  uint32_t* r1;
  uint32_t* challenges;
};
cudaError_t launch_sumcheck(const uint32_t* evals, uint32_t log_n, uint32_t* scratch, SumcheckOut* out, cudaStream_t s);
}  // namespace azk

using namespace azk;

namespace {

struct InstanceCfg {
  uint32_t logn, rounds, queries, log_blowup, grinding;
  std::vector<uint64_t> claimed;
  uint32_t leaf_values = 1;  // QM31 values per Merkle leaf: 1 (16-byte leaves) or 4 (64-byte leaves)
};

struct Engine {
  azk_ctx* ctx = nullptr;
  cudaStream_t s = nullptr;
  // Uploads (input copies and the scan launch) run on a high-priority stream: their
  // one launch takes the first free SM slots instead of queueing behind another
  // prover's superstep, so one prover uploads while another proves.
  cudaStream_t s_up = nullptr;
  bool owns_streams = true;
  Sched sched;
  std::vector<InstanceCfg> cfg;
  uint32_t rmax = 0, qmax = 0;
  bool any_grinding = false;

  Arena arena;
  std::vector<uint64_t> off_input, off_layers, off_trees, off_tr, off_ch, off_cm, off_qp, off_claim, off_proof, off_cnt;
  std::vector<uint64_t> proof_len, proof_off;
  uint64_t proof_total = 0;
  uint64_t off_inst = 0, off_flag = 0, off_info = 0;

  std::vector<PcsInstance> h_inst;
  // FFT
  uint32_t leaf_values = 1;  // all instances of an engine share the leaf size
  FftPlan fft;
  std::vector<FftJob> fft_transforms;
  DevBuf d_scan;  // upload scan jobs, one per instance
  std::vector<uint8_t> fft_narrow;  // per instance: input known to be a lifted M31 polynomial
  // rounds: tree step k (kind QM31 at k == 0, fold+hash after), final folds at step k
  std::vector<TreeJob> tree_jobs;
  std::vector<uint2> tree_work;
  std::vector<uint64_t> tstep_off, tstep_cnt;
  std::vector<std::vector<std::pair<uint64_t, uint64_t>>> tstep_inst;  // [step][inst]
  std::vector<uint32_t> tstep_tile;                                     // max tile log per step
  std::vector<FoldJob> fold_jobs;
  std::vector<uint2> fold_work;
  std::vector<uint64_t> fstep_off, fstep_cnt;
  std::vector<std::vector<std::pair<uint64_t, uint64_t>>> fstep_inst;
  std::vector<uint32_t> ids;
  DevBuf d_tree_jobs, d_tree_work, d_fold_jobs, d_fold_work, d_ids;

  cudaGraphExec_t graph = nullptr;
  bool graph_from_coeffs = false;

  // Per-stage CUDA events (profiling): stage kind 0 = FFT, 1 = tree (fold +
  // hash + transcript), 2 = final fold, 3 = transcript/queries/emission.
  bool prof = false;
  std::vector<int> ev_kind;
  std::vector<cudaEvent_t> ev_a, ev_b;
  size_t ev_used = 0;
  // algorithmic work per superstep
  uint64_t tree_perms = 0, fft_bytes = 0, fold_bytes = 0;
  uint32_t launches = 0;

  ~Engine() {
    if (graph) cudaGraphExecDestroy(graph);
    for (auto e : ev_a) cudaEventDestroy(e);
    for (auto e : ev_b) cudaEventDestroy(e);
    if (owns_streams && s) cudaStreamDestroy(s);
    if (owns_streams && s_up) cudaStreamDestroy(s_up);
  }

  // Event pair for the next profiled region (created up front, outside capture).
  void ensure_events(size_t n) {
    while (ev_a.size() < n) {
      cudaEvent_t a, b;
      AZK_CU(cudaEventCreate(&a));
      AZK_CU(cudaEventCreate(&b));
      ev_a.push_back(a);
      ev_b.push_back(b);
      ev_kind.push_back(0);
    }
  }
  void prof_begin(int kind) {
    if (!prof) return;
    ev_kind[ev_used] = kind;
    AZK_CU(cudaEventRecord(ev_a[ev_used], s));
  }
  void prof_end() {
    if (!prof) return;
    AZK_CU(cudaEventRecord(ev_b[ev_used], s));
    ev_used++;
  }
  void profile(double* sec) {
    for (int k = 0; k < 4; k++) sec[k] = 0;
    for (size_t i = 0; i < ev_used; i++) {
      float ms = 0;
      AZK_CU(cudaEventElapsedTime(&ms, ev_a[i], ev_b[i]));
      sec[ev_kind[i]] += ms / 1000.0;
    }
  }

  PcsInstance* d_inst() const { return arena.at<PcsInstance>(off_inst); }
  uint32_t* d_flag() const { return arena.at<uint32_t>(off_flag); }
  InputInfo* d_info() const { return arena.at<InputInfo>(off_info); }

  // Canonicality gate over the staged coefficients of every instance (counts[i]
  // leading QM31 values; the rest are zero) and the FFT's input description:
  // which instances are lifted M31 polynomials, how many coefficients are nonzero.
  // Gate and describe the uploaded coefficients (the caller queued their copies
  // on s_up): canonicality, the lifted-M31 flag and zeros over each tail
  // [counts[i], N) in one launch on s_up, then one small readback.
  void scan_inputs(const std::vector<uint64_t>& counts) {
    std::vector<InputInfo> h(cfg.size());
    for (size_t i = 0; i < cfg.size(); i++) h[i] = InputInfo{1u, 0u, counts[i]};
    AZK_CU(cudaMemcpyAsync(d_info(), h.data(), sizeof(InputInfo) * h.size(), cudaMemcpyHostToDevice, s_up));
    AZK_CU(cudaMemsetAsync(d_flag(), 0, 4, s_up));
    std::vector<ScanJob> jobs(cfg.size());
    uint64_t max_n = 0;
    for (size_t i = 0; i < cfg.size(); i++) {
      const uint64_t N = 1ull << cfg[i].logn;
      jobs[i] = ScanJob{arena.at<uint4>(off_input[i]), counts[i], N, d_info() + i};
      max_n = std::max(max_n, N);
    }
    if (!d_scan.p) d_scan.alloc(sizeof(ScanJob) * cfg.size(), "PCS.ScanJobs");
    AZK_CU(cudaMemcpyAsync(d_scan.p, jobs.data(), sizeof(ScanJob) * jobs.size(), cudaMemcpyHostToDevice, s_up));
    AZK_CU(launch_scan_inputs(d_scan.as<ScanJob>(), (uint32_t)jobs.size(), max_n, d_flag(), s_up));
    uint32_t f = 0;
    AZK_CU(cudaMemcpyAsync(&f, d_flag(), 4, cudaMemcpyDeviceToHost, s_up));
    AZK_CU(cudaMemcpyAsync(h.data(), d_info(), sizeof(InputInfo) * h.size(), cudaMemcpyDeviceToHost, s_up));
    sync_stream(s_up);
    layout(f == 0, "input contains a non-canonical field element");
    std::vector<uint8_t> narrow(cfg.size());
    for (size_t i = 0; i < cfg.size(); i++) narrow[i] = h[i].m31 ? 1 : 0;
    set_fft_narrow(narrow);
  }
  // Inputs written by the caller through a device pointer: nothing known.
  void forget_input(size_t i) {
    AZK_CU(cudaMemsetAsync(d_info() + i, 0, sizeof(InputInfo), s));
    std::vector<uint8_t> narrow = fft_narrow;
    narrow[i] = 0;
    set_fft_narrow(narrow);
  }
  // Which instances run the one-limb FFT kernel; a change rebuilds the FFT work
  // lists and drops the captured graph (it is captured again on the next run).
  void set_fft_narrow(const std::vector<uint8_t>& narrow) {
    if (narrow == fft_narrow) return;
    sync_stream(s);
    fft_narrow = narrow;
    fft.build(fft_transforms, fft_narrow);
    fft.upload(s);
    sync_stream(s);
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
  }

  // `run_stream` / `upload_stream`: streams owned by the caller (a server worker,
  // whose engines never run at the same time), else the engine creates its own.
  void init(azk_ctx* c, const std::vector<InstanceCfg>& cf, const Sched& sc, cudaStream_t run_stream = nullptr,
            cudaStream_t upload_stream = nullptr) {
    ctx = c;
    sched = sc;
    cfg = cf;
    AZK_CU(cudaSetDevice(ctx->device));
    if (run_stream && upload_stream) {
      s = run_stream;
      s_up = upload_stream;
      owns_streams = false;
    } else {
      AZK_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      int prio_lo = 0, prio_hi = 0;
      AZK_CU(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
      AZK_CU(cudaStreamCreateWithPriority(&s_up, cudaStreamNonBlocking, prio_hi));
    }
    size_t n = cfg.size();
    leaf_values = cfg.empty() ? 1 : cfg[0].leaf_values;
    for (auto& i : cfg) {
      layout(i.leaf_values == leaf_values && (leaf_values == 1 || leaf_values == 4), "all instances of a batch share one leaf size (16 or 64 bytes)");
      // a 64-byte leaf holds 4 values: every committed layer needs at least 4
      layout(leaf_values == 1 || i.logn >= i.rounds + 1, "64-byte leaves need at least 4 values in every committed layer");
      rmax = std::max(rmax, i.rounds);
      qmax = std::max(qmax, i.queries);
      any_grinding |= i.grinding > 0;
    }
    // ---- memory plan ----
    auto resz = [&](std::vector<uint64_t>& v) { v.assign(n, 0); };
    for (auto* v : {&off_input, &off_layers, &off_trees, &off_tr, &off_ch, &off_cm, &off_qp, &off_claim, &off_proof, &off_cnt}) resz(*v);
    proof_len.assign(n, 0);
    proof_off.assign(n, 0);
    for (size_t i = 0; i < n; i++) {
      const auto& c2 = cfg[i];
      uint64_t N = 1ull << c2.logn;
      off_input[i] = arena.reserve(16 * N);
      off_layers[i] = arena.reserve(16 * 2 * N);
      off_trees[i] = arena.reserve(32 * 2 * N);
      off_tr[i] = arena.reserve(sizeof(Transcript));
      off_ch[i] = arena.reserve(16ull * c2.rounds);
      off_cm[i] = arena.reserve(32ull * c2.rounds);
      off_qp[i] = arena.reserve(4ull * c2.queries);
      off_claim[i] = arena.reserve(8ull * c2.claimed.size());
      off_cnt[i] = arena.reserve(4 * tree_counter_count(c2.logn, 1));
      proof_len[i] = c2.leaf_values == 1 ? proof_total_bytes(c2.logn, c2.rounds, c2.queries, (uint32_t)c2.claimed.size(), c2.grinding > 0) : 0;
    }
    uint64_t pbase = arena.reserve(0);
    arena.used = pbase;
    for (size_t i = 0; i < n; i++) {
      proof_off[i] = proof_total;
      proof_total += align_up(proof_len[i], 16);
    }
    uint64_t off_proofs = arena.reserve(proof_total);
    for (size_t i = 0; i < n; i++) off_proof[i] = off_proofs + proof_off[i];
    off_inst = arena.reserve(sizeof(PcsInstance) * n);
    off_flag = arena.reserve(16);
    off_info = arena.reserve(sizeof(InputInfo) * n);
    arena.commit("PCS.Arena");
    // counters and inputs start at zero
    AZK_CU(cudaMemsetAsync(arena.buf.p, 0, arena.used, s));

    // ---- instance table ----
    h_inst.resize(n);
    for (size_t i = 0; i < n; i++) {
      const auto& c2 = cfg[i];
      const auto& dom = domain_tables(ctx, c2.logn);
      PcsInstance& I = h_inst[i];
      I = PcsInstance{};
      I.logn = c2.logn;
      I.rounds = c2.rounds;
      I.queries = c2.queries;
      I.log_blowup = c2.log_blowup;
      I.grinding_bits = c2.grinding;
      I.n_claimed = (uint32_t)c2.claimed.size();
      I.layers = arena.at<uint4>(off_layers[i]);
      I.trees = arena.at<uint64_t>(off_trees[i]);
      I.tw = dom.tw;
      I.inv = dom.inv;
      I.transcript = arena.at<Transcript>(off_tr[i]);
      I.challenges = arena.at<uint32_t>(off_ch[i]);
      I.commitments = arena.at<uint64_t>(off_cm[i]);
      I.query_pairs = arena.at<uint32_t>(off_qp[i]);
      I.claimed = arena.at<uint64_t>(off_claim[i]);
      I.proof = arena.at<uint8_t>(off_proof[i]);
      I.proof_len = proof_len[i];
      if (!c2.claimed.empty())
        AZK_CU(cudaMemcpyAsync(arena.at<uint64_t>(off_claim[i]), c2.claimed.data(), 8 * c2.claimed.size(), cudaMemcpyHostToDevice, s));
    }
    AZK_CU(cudaMemcpyAsync(d_inst(), h_inst.data(), sizeof(PcsInstance) * n, cudaMemcpyHostToDevice, s));
    ids.resize(n);
    for (size_t i = 0; i < n; i++) ids[i] = (uint32_t)i;
    d_ids.alloc(4 * n, "PCS.Ids");
    AZK_CU(cudaMemcpyAsync(d_ids.p, ids.data(), 4 * n, cudaMemcpyHostToDevice, s));

    // ---- FFT ----
    std::vector<FftJob> tf;
    for (size_t i = 0; i < n; i++)
      tf.push_back(FftJob{cfg[i].logn, 0, arena.at<uint4>(off_input[i]), arena.at<uint4>(off_layers[i]), h_inst[i].tw,
                          arena.at<uint32_t>(off_trees[i]), d_info() + i});
    fft_transforms = tf;
    fft_narrow.assign(n, 0);
    fft.build(tf, fft_narrow);
    fft.upload(s);

    // ---- rounds ----
    tstep_off.assign(rmax, 0);
    tstep_cnt.assign(rmax, 0);
    tstep_tile.assign(rmax, 1);
    tstep_inst.assign(rmax, std::vector<std::pair<uint64_t, uint64_t>>(n, {0, 0}));
    fstep_off.assign(rmax + 1, 0);
    fstep_cnt.assign(rmax + 1, 0);
    fstep_inst.assign(rmax + 1, std::vector<std::pair<uint64_t, uint64_t>>(n, {0, 0}));
    // large instances first inside a step, so their upper-tree tails overlap the rest
    std::vector<uint32_t> order(n);
    for (size_t i = 0; i < n; i++) order[i] = (uint32_t)i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cfg[a].logn > cfg[b].logn; });
    for (uint32_t k = 0; k < rmax; k++) {
      tstep_off[k] = tree_work.size();
      for (uint32_t i : order) {
        const auto& c2 = cfg[i];
        if (k >= c2.rounds) continue;
        const PcsInstance& I = h_inst[i];
        // leaves of layer k: 2^(logn - k) values, one or four per leaf
        uint32_t lg = c2.logn - k - (leaf_values == 4 ? 2 : 0);
        uint32_t tl = tree_tile_log(sched, lg);
        if (tl == 0 && lg > 0) tl = 1;
        TreeJob j{};
        j.logn = lg;
        j.kind = tree_kind(k);
        j.tile_log = tl;
        j.group_log = std::max<uint32_t>(1, std::min(sched.group_log, tl));
        if (k == 0) {
          j.layer = I.layers;
        } else {
          j.layer = I.layers + layer_offset(c2.logn, k - 1);
          j.inv = I.inv + (k - 1 == 0 ? 0 : (1ull << c2.logn) - ((1ull << c2.logn) >> (k - 1)));
          j.fold_ch = I.challenges + 4 * (k - 1);
          j.out_layer = I.layers + layer_offset(c2.logn, k);
        }
        j.inner = I.trees + 4 * tree_offset(c2.logn, k);
        j.counters = arena.at<uint32_t>(off_cnt[i]);
        j.root_action = kRootCircleRound;
        j.round = k;
        j.transcript = I.transcript;
        j.challenge_out = I.challenges + 4 * k;
        j.root_out = I.commitments + 4 * k;
        uint32_t jid = (uint32_t)tree_jobs.size();
        tree_jobs.push_back(j);
        uint64_t tiles = 1ull << (lg - tl);
        tstep_inst[k][i] = {tree_work.size(), tiles};
        for (uint64_t t = 0; t < tiles; t++) tree_work.push_back(make_uint2(jid, (uint32_t)t));
        tstep_tile[k] = std::max(tstep_tile[k], tl);
      }
      tstep_cnt[k] = tree_work.size() - tstep_off[k];
    }
    for (uint32_t k = 1; k <= rmax; k++) {
      fstep_off[k] = fold_work.size();
      for (uint32_t i : order) {
        const auto& c2 = cfg[i];
        if (c2.rounds != k) continue;
        const PcsInstance& I = h_inst[i];
        uint64_t N = 1ull << c2.logn;
        FoldJob f{N >> k, I.layers + layer_offset(c2.logn, k - 1), I.inv + (k - 1 == 0 ? 0 : N - (N >> (k - 1))), I.challenges + 4 * (k - 1),
                  I.layers + layer_offset(c2.logn, k)};
        uint32_t fid = (uint32_t)fold_jobs.size();
        fold_jobs.push_back(f);
        uint64_t chunks = (f.n_out + kFoldChunk - 1) / kFoldChunk;
        fstep_inst[k][i] = {fold_work.size(), chunks};
        for (uint64_t c3 = 0; c3 < chunks; c3++) fold_work.push_back(make_uint2(fid, (uint32_t)c3));
      }
      fstep_cnt[k] = fold_work.size() - fstep_off[k];
    }
    auto up = [&](DevBuf& d, const void* src, size_t bytes, const char* label) {
      d.alloc(std::max<size_t>(bytes, 16), label);
      if (bytes) AZK_CU(cudaMemcpyAsync(d.p, src, bytes, cudaMemcpyHostToDevice, s));
    };
    up(d_tree_jobs, tree_jobs.data(), tree_jobs.size() * sizeof(TreeJob), "PCS.TreeJobs");
    up(d_tree_work, tree_work.data(), tree_work.size() * sizeof(uint2), "PCS.TreeWork");
    up(d_fold_jobs, fold_jobs.data(), fold_jobs.size() * sizeof(FoldJob), "PCS.FoldJobs");
    up(d_fold_work, fold_work.data(), fold_work.size() * sizeof(uint2), "PCS.FoldWork");
    sync_stream(s);
    // algorithmic work: leaf + parent permutations and 3 transcript absorbs per
    // committed layer; FFT single-pass bytes (16N in, 16N out, 4(N-1) twiddles);
    // final fold bytes (16 in + 8 out + 2 twiddle per input element)
    for (auto& c2 : cfg) {
      uint64_t N = 1ull << c2.logn;
      for (uint32_t k = 0; k < c2.rounds; k++) tree_perms += 2 * (N >> k) - 1 + 3;
      fft_bytes += 32 * N + 4 * (N - 1);
      fold_bytes += 26 * (N >> (c2.rounds - 1));
    }
    launches = 0;
    for (auto c3 : fft.step_cnt) launches += c3 ? 1 : 0;
    for (auto c3 : tstep_cnt) launches += c3 ? 1 : 0;
    for (auto c3 : fstep_cnt) launches += c3 ? 1 : 0;
    launches += 4;  // prefix, finalize, queries, emit
    ensure_events(fft.step_cnt.size() + 2 * rmax + 8);
  }

  uint32_t tree_kind(uint32_t k) const {
    if (leaf_values == 4) return k == 0 ? kLeafQM31x4 : kLeafFoldx4;
    return k == 0 ? kLeafQM31 : kLeafFold;
  }
  void launch_tree_range(uint32_t k, uint64_t off, uint64_t cnt) {
    if (!cnt) return;
    AZK_CU(launch_tree_jobs(d_tree_jobs.as<TreeJob>(), d_tree_work.as<uint2>() + off, (uint32_t)cnt, tstep_tile[k], tree_kind(k), sched.threads, s));
  }
  void launch_fold_range(uint64_t off, uint64_t cnt) {
    if (!cnt) return;
    AZK_CU(launch_fold_jobs(d_fold_jobs.as<FoldJob>(), d_fold_work.as<uint2>() + off, (uint32_t)cnt, s));
  }

  // Everything up to (not including) grinding.  from_coeffs: run the FFT first.
  void enqueue_rounds_batched(bool from_coeffs) {
    ev_used = 0;
    if (from_coeffs) {
      for (size_t st = 0; st < fft.step_cnt.size(); st++) {
        prof_begin(0);
        fft.launch_step(st, s);
        prof_end();
      }
    }
    prof_begin(3);
    AZK_CU(launch_pcs_prefix(d_inst(), (uint32_t)cfg.size(), s));
    prof_end();
    for (uint32_t k = 0; k <= rmax; k++) {
      if (k < rmax) {
        prof_begin(1);
        launch_tree_range(k, tstep_off[k], tstep_cnt[k]);
        prof_end();
      }
      if (k >= 1 && fstep_cnt[k]) {
        prof_begin(2);
        launch_fold_range(fstep_off[k], fstep_cnt[k]);
        prof_end();
      }
    }
    prof_begin(3);
    AZK_CU(launch_pcs_finalize(d_inst(), d_ids.as<uint32_t>(), (uint32_t)cfg.size(), s));
    prof_end();
  }
  // Proof bytes exist only for 16-byte leaves (the reference's verifier opens one
  // QM31 value per leaf); a 64-byte-leaf chain ends with its final layer.
  bool has_proofs() const { return leaf_values == 1; }
  void enqueue_tail_batched() {
    if (!has_proofs()) return;
    prof_begin(3);
    AZK_CU(launch_pcs_queries(d_inst(), d_ids.as<uint32_t>(), (uint32_t)cfg.size(), s));
    AZK_CU(launch_pcs_emit(d_inst(), d_ids.as<uint32_t>(), (uint32_t)cfg.size(), qmax, s));
    prof_end();
  }
  void enqueue_instance(uint32_t i, bool from_coeffs) {
    if (from_coeffs)
      for (size_t st = 0; st < fft.step_cnt.size(); st++)
        if (fft.inst_range[st][i].second) fft.launch_step_for(st, i, s);
    AZK_CU(launch_pcs_prefix(d_inst() + i, 1, s));
    const uint32_t* id = d_ids.as<uint32_t>() + i;
    for (uint32_t k = 0; k <= cfg[i].rounds; k++) {
      if (k < cfg[i].rounds) launch_tree_range(k, tstep_inst[k][i].first, tstep_inst[k][i].second);
      if (k == cfg[i].rounds) launch_fold_range(fstep_inst[k][i].first, fstep_inst[k][i].second);
    }
    AZK_CU(launch_pcs_finalize(d_inst(), id, 1, s));
    if (!has_proofs()) return;
    grind_instance(i);
    AZK_CU(launch_pcs_queries(d_inst(), id, 1, s));
    AZK_CU(launch_pcs_emit(d_inst(), id, 1, cfg[i].queries, s));
  }

  // Smallest nonce meeting the grinding target (CircleProofFormat.swift:753-794),
  // searched in increasing chunks on the device.
  void grind_instance(uint32_t i) {
    if (!cfg[i].grinding) return;
    DevBuf found(8, "PCS.GrindingNonce");
    uint64_t chunk = 1ull << std::min<uint32_t>(cfg[i].grinding + 4, 26);
    for (uint64_t start = 0;; start += chunk) {
      AZK_CU(cudaMemsetAsync(found.p, 0xFF, 8, s));
      AZK_CU(launch_pcs_grind(d_inst(), i, start, chunk, found.as<unsigned long long>(), s));
      uint64_t nonce = ~0ull;
      AZK_CU(cudaMemcpyAsync(&nonce, found.p, 8, cudaMemcpyDeviceToHost, s));
      sync_stream(s);
      if (nonce != ~0ull) {
        h_inst[i].nonce = nonce;
        h_inst[i].has_nonce = 1;
        AZK_CU(cudaMemcpyAsync(&d_inst()[i].nonce, &h_inst[i].nonce, 8, cudaMemcpyHostToDevice, s));
        AZK_CU(cudaMemcpyAsync(&d_inst()[i].has_nonce, &h_inst[i].has_nonce, 4, cudaMemcpyHostToDevice, s));
        return;
      }
      require(start < (1ull << 40), AZK_ERR_COMMAND_EXECUTION_FAILED, "grinding nonce search exhausted");
    }
  }

  void set_publics(const uint8_t* pubs) {
    for (size_t i = 0; i < cfg.size(); i++) std::memcpy(h_inst[i].pub, pubs + 32 * i, 32);
    AZK_CU(cudaMemcpy2DAsync(reinterpret_cast<uint8_t*>(d_inst()) + offsetof(PcsInstance, pub), sizeof(PcsInstance), pubs, 32, 32, cfg.size(),
                             cudaMemcpyHostToDevice, s));
  }

  // Run the whole superstep; returns device seconds.
  double run(bool from_coeffs, bool plain, uint64_t* submit_ns, const Timer& t) {
    AZK_CU(cudaMemsetAsync(d_flag(), 0, 4, s));
    GpuTimer g(s);
    if (plain) {
      ev_used = 0;
      for (uint32_t i = 0; i < cfg.size(); i++) enqueue_instance(i, from_coeffs);
    } else if (!any_grinding && sched.graph && !prof) {
      // (profiled runs take the eager path below: the same launch sequence, with
      // event pairs around each stage)
      if (!graph || graph_from_coeffs != from_coeffs) {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        cudaGraph_t gr;
        AZK_CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue_rounds_batched(from_coeffs);
        enqueue_tail_batched();
        AZK_CU(cudaStreamEndCapture(s, &gr));
        AZK_CU(cudaGraphInstantiate(&graph, gr, 0));
        cudaGraphDestroy(gr);
        graph_from_coeffs = from_coeffs;
      }
      AZK_CU(cudaGraphLaunch(graph, s));
    } else {
      enqueue_rounds_batched(from_coeffs);
      for (uint32_t i = 0; i < cfg.size(); i++) grind_instance(i);
      enqueue_tail_batched();
    }
    if (submit_ns) *submit_ns = t.ns();
    g.stop();
    return g.seconds();
  }

  // Reject non-canonical inputs (QM31CanonicalityCheck.swift): checked on the
  // device before the proof is trusted.
  void check_input_canonical(const void* dptr, uint64_t words) {
    AZK_CU(cudaMemsetAsync(d_flag(), 0, 4, s));
    AZK_CU(launch_check_canonical(static_cast<const uint32_t*>(dptr), words, d_flag(), s));
    uint32_t f = 0;
    AZK_CU(cudaMemcpyAsync(&f, d_flag(), 4, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
    layout(f == 0, "input contains a non-canonical field element");
  }

  void trace(uint32_t i, uint8_t* cm, uint32_t* ch, uint32_t* fl, uint32_t* qp) {
    const auto& c2 = cfg[i];
    if (cm) AZK_CU(cudaMemcpyAsync(cm, arena.at<uint8_t>(off_cm[i]), 32ull * c2.rounds, cudaMemcpyDeviceToHost, s));
    if (ch) AZK_CU(cudaMemcpyAsync(ch, arena.at<uint8_t>(off_ch[i]), 16ull * c2.rounds, cudaMemcpyDeviceToHost, s));
    if (fl)
      AZK_CU(cudaMemcpyAsync(fl, h_inst[i].layers + layer_offset(c2.logn, c2.rounds), 16ull << (c2.logn - c2.rounds), cudaMemcpyDeviceToHost, s));
    if (qp) AZK_CU(cudaMemcpyAsync(qp, arena.at<uint8_t>(off_qp[i]), 4ull * c2.queries, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
  }
};

void validate_params(uint32_t logn, uint32_t log_blowup, uint32_t queries, uint32_t grinding, uint32_t rounds) {
  // CircleFRISecurityParametersV1.init (CircleProofFormat.swift:136-151) and
  // CircleFRIProofBuilderV1.prove (CircleProofFormat.swift:1181-1189)
  layout(logn >= 1 && logn <= 26);
  layout(log_blowup > 0 && queries > 0 && grinding <= 20);
  layout((uint64_t)log_blowup * queries + grinding <= 0xFFFFFFFFull);
  layout(rounds >= 1 && rounds <= logn);
}

}  // namespace

struct azk_pcs_prover {
  azk_ctx* ctx;
  std::mutex mu;
  Engine eng;
  uint32_t logn, rounds, queries, log_blowup, grinding;
};

struct azk_batch {
  azk_ctx* ctx;
  std::mutex mu;
  Engine eng;
};

extern "C" {

uint64_t azk_pcs_proof_size(uint32_t logn, uint32_t rounds, uint32_t queries, uint32_t claimed, uint32_t grinding) {
  if (logn < 1 || logn > 30 || rounds < 1 || rounds > logn) return 0;
  return proof_total_bytes(logn, rounds, queries, claimed, grinding > 0);
}

azk_status azk_pcs_prover_create(azk_ctx* ctx, uint32_t logn, uint32_t log_blowup, uint32_t queries, uint32_t grinding, uint32_t rounds,
                                 const azk_schedule* schedule, azk_pcs_prover** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    validate_params(logn, log_blowup, queries, grinding, rounds);
    auto p = std::make_unique<azk_pcs_prover>();
    p->ctx = ctx;
    p->logn = logn;
    p->rounds = rounds;
    p->queries = queries;
    p->log_blowup = log_blowup;
    p->grinding = grinding;
    Sched sc = resolve_schedule(schedule, kTuned_pcs_single);
    sc.graph = false;
    p->eng.init(ctx, {InstanceCfg{logn, rounds, queries, log_blowup, grinding, {}}}, sc);
    *out = p.release();
  });
}

// Claimed openings change the proof layout: rebuild the engine for a new set
// before any input is staged into it.
static void pcs_ensure_claimed(azk_pcs_prover* p, const std::vector<uint64_t>& claimed) {
  Engine& e = p->eng;
  if (claimed == e.cfg[0].claimed) return;
  Sched sc = e.sched;
  e.~Engine();
  new (&e) Engine();
  e.init(p->ctx, {InstanceCfg{p->logn, p->rounds, p->queries, p->log_blowup, p->grinding, claimed}}, sc);
}

static void pcs_prove_common(azk_pcs_prover* p, bool coeffs, const uint8_t pub[32], uint8_t* proof_out, bool proof_on_device, uint64_t* proof_len,
                             azk_stats* st, const Timer& t) {
  Engine& e = p->eng;
  e.set_publics(pub);
  uint64_t sub = 0;
  double gs = e.run(coeffs, true, &sub, t);
  uint64_t len = e.proof_len[0];
  layout(*proof_len >= len, "proof buffer too small");
  *proof_len = len;
  if (proof_on_device)
    AZK_CU(cudaMemcpyAsync(proof_out, e.h_inst[0].proof, len, cudaMemcpyDeviceToDevice, e.s));
  else
    AZK_CU(cudaMemcpyAsync(proof_out, e.h_inst[0].proof, len, cudaMemcpyDeviceToHost, e.s));
  sync_stream(e.s);
  fill_stats(st, t, sub, gs);
}

azk_status azk_pcs_prover_prove_evaluations(azk_pcs_prover* p, const uint32_t* ev, const uint8_t pub[32], const uint64_t* claimed, uint64_t nclaimed,
                                            uint8_t* proof_out, uint64_t* proof_len, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && ev && pub && proof_out && proof_len && (claimed || !nclaimed));
    std::lock_guard<std::mutex> lk(p->mu);
    uint64_t N = 1ull << p->logn;
    std::vector<uint64_t> cl(claimed, claimed + nclaimed);
    std::sort(cl.begin(), cl.end());
    for (size_t i = 0; i < cl.size(); i++) layout(cl[i] < N && (i == 0 || cl[i - 1] < cl[i]));
    Timer t;
    pcs_ensure_claimed(p, cl);
    Engine& e = p->eng;
    // evaluations go straight into layer 0
    AZK_CU(cudaMemcpyAsync(e.h_inst[0].layers, ev, 16 * N, cudaMemcpyHostToDevice, e.s));
    e.check_input_canonical(e.h_inst[0].layers, 4 * N);
    pcs_prove_common(p, false, pub, proof_out, false, proof_len, st, t);
  });
}

azk_status azk_pcs_prover_prove_coefficients(azk_pcs_prover* p, const uint32_t* coeffs, uint64_t count, const uint8_t pub[32], uint8_t* proof_out,
                                             uint64_t* proof_len, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && coeffs && pub && proof_out && proof_len);
    std::lock_guard<std::mutex> lk(p->mu);
    uint64_t N = 1ull << p->logn;
    layout(count >= 1 && count <= N);
    Timer t;
    pcs_ensure_claimed(p, {});
    Engine& e = p->eng;
    uint4* in = e.arena.at<uint4>(e.off_input[0]);
    AZK_CU(cudaMemcpyAsync(in, coeffs, 16 * count, cudaMemcpyHostToDevice, e.s_up));
    e.scan_inputs({count});
    pcs_prove_common(p, true, pub, proof_out, false, proof_len, st, t);
  });
}

azk_status azk_pcs_prover_prove_resident(azk_pcs_prover* p, const void* din, uint64_t in_off, int is_coeffs, const uint8_t pub[32], void* dproof,
                                         uint64_t* proof_len, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && din && pub && dproof && proof_len && in_off % 16 == 0);
    std::lock_guard<std::mutex> lk(p->mu);
    uint64_t N = 1ull << p->logn;
    Timer t;
    pcs_ensure_claimed(p, {});
    Engine& e = p->eng;
    const uint8_t* src = static_cast<const uint8_t*>(din) + in_off;
    void* dst = is_coeffs ? (void*)e.arena.at<uint4>(e.off_input[0]) : (void*)e.h_inst[0].layers;
    if (is_coeffs) {
      AZK_CU(cudaMemcpyAsync(dst, src, 16 * N, cudaMemcpyDeviceToDevice, e.s_up));
      e.scan_inputs({N});
    } else {
      AZK_CU(cudaMemcpyAsync(dst, src, 16 * N, cudaMemcpyDeviceToDevice, e.s));
      e.check_input_canonical(dst, 4 * N);
    }
    pcs_prove_common(p, is_coeffs != 0, pub, static_cast<uint8_t*>(dproof), true, proof_len, st, t);
  });
}

azk_status azk_pcs_prover_trace(azk_pcs_prover* p, uint8_t* cm, uint32_t* ch, uint32_t* fl, uint32_t* qp) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    p->eng.trace(0, cm, ch, fl, qp);
  });
}

void azk_pcs_prover_destroy(azk_pcs_prover* p) { delete p; }

azk_status azk_circle_merkle_fold_chain(azk_ctx* ctx, uint32_t logn, const uint32_t* ev, uint32_t log_blowup, uint32_t queries, uint32_t grinding,
                                        const uint8_t pub[32], uint32_t rounds, uint32_t* final_out, uint8_t* cm_out, uint32_t* ch_out, azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && ev && pub && final_out);
    validate_params(logn, log_blowup, queries, grinding, rounds);
    uint64_t N = 1ull << logn;
    Timer t;
    Engine e;
    Sched sc = resolve_schedule(nullptr, kTuned_pcs_single);
    sc.graph = false;
    e.init(ctx, {InstanceCfg{logn, rounds, queries, log_blowup, grinding, {}}}, sc);
    AZK_CU(cudaMemcpyAsync(e.h_inst[0].layers, ev, 16 * N, cudaMemcpyHostToDevice, e.s));
    e.check_input_canonical(e.h_inst[0].layers, 4 * N);
    e.set_publics(pub);
    GpuTimer g(e.s);
    AZK_CU(launch_pcs_prefix(e.d_inst(), 1, e.s));
    for (uint32_t k = 0; k <= rounds; k++) {
      if (k < rounds) e.launch_tree_range(k, e.tstep_inst[k][0].first, e.tstep_inst[k][0].second);
      if (k == rounds) e.launch_fold_range(e.fstep_inst[k][0].first, e.fstep_inst[k][0].second);
    }
    g.stop();
    double gs = g.seconds();
    e.trace(0, cm_out, ch_out, final_out, nullptr);
    fill_stats(st, t, 0, gs);
  });
}

// ---- batch ----
azk_status azk_batch_create_leaves(azk_ctx* ctx, uint32_t count, const uint32_t* logs, const uint32_t* rounds, uint32_t log_blowup, uint32_t queries,
                                   uint32_t leaf_bytes, const azk_schedule* schedule, azk_batch** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && logs && rounds && count >= 1);
    layout(leaf_bytes == 16 || leaf_bytes == 64, "leaf_bytes must be 16 (one QM31 per leaf) or 64 (four)");
    std::vector<InstanceCfg> cf;
    for (uint32_t i = 0; i < count; i++) {
      validate_params(logs[i], log_blowup, queries, 0, rounds[i]);
      cf.push_back(InstanceCfg{logs[i], rounds[i], queries, log_blowup, 0, {}, leaf_bytes / 16});
    }
    auto b = std::make_unique<azk_batch>();
    b->ctx = ctx;
    b->eng.init(ctx, cf, resolve_schedule(schedule, kTuned_pcs_batch));
    *out = b.release();
  });
}

azk_status azk_batch_create(azk_ctx* ctx, uint32_t count, const uint32_t* logs, const uint32_t* rounds, uint32_t log_blowup, uint32_t queries,
                            const azk_schedule* schedule, azk_batch** out) {
  return azk_batch_create_leaves(ctx, count, logs, rounds, log_blowup, queries, 16, schedule, out);
}

azk_status azk_batch_input(azk_batch* b, uint32_t i, void** dev) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b && dev && i < b->eng.cfg.size());
    std::lock_guard<std::mutex> lk(b->mu);
    // the caller writes this input directly: what the last upload learned about it
    // no longer holds (the FFT reads all N coefficients with QM31 arithmetic)
    b->eng.forget_input(i);
    sync_stream(b->eng.s);
    *dev = b->eng.arena.at<void>(b->eng.off_input[i]);
  });
}

azk_status azk_batch_upload(azk_batch* b, const uint32_t* host, const uint64_t* offsets, const uint64_t* counts) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b && host && offsets && counts);
    std::lock_guard<std::mutex> lk(b->mu);
    Engine& e = b->eng;
    for (size_t i = 0; i < e.cfg.size(); i++) {
      uint64_t N = 1ull << e.cfg[i].logn;
      layout(counts[i] >= 1 && counts[i] <= N);
      uint4* in = e.arena.at<uint4>(e.off_input[i]);
      AZK_CU(cudaMemcpyAsync(in, host + 4 * offsets[i], 16 * counts[i], cudaMemcpyHostToDevice, e.s_up));
    }
    // every staged word must be canonical (QM31CanonicalityCheck.swift:11-117)
    e.scan_inputs(std::vector<uint64_t>(counts, counts + e.cfg.size()));
  });
}

azk_status azk_batch_prove(azk_batch* b, const uint8_t* pubs, int plain, azk_stats* st) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b && pubs);
    std::lock_guard<std::mutex> lk(b->mu);
    Timer t;
    Engine& e = b->eng;
    e.set_publics(pubs);
    uint64_t sub = 0;
    double gs = e.run(true, plain != 0, &sub, t);
    sync_stream(e.s);
    fill_stats(st, t, sub, gs);
  });
}

azk_status azk_batch_proof_sizes(azk_batch* b, uint64_t* sizes, uint64_t* total) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b != nullptr);
    uint64_t tt = 0;
    for (size_t i = 0; i < b->eng.cfg.size(); i++) {
      if (sizes) sizes[i] = b->eng.proof_len[i];
      tt += b->eng.proof_len[i];
    }
    if (total) *total = tt;
  });
}

azk_status azk_batch_download_proofs(azk_batch* b, uint8_t* out, uint64_t cap) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b && out);
    std::lock_guard<std::mutex> lk(b->mu);
    Engine& e = b->eng;
    layout(e.has_proofs(), "a 64-byte-leaf batch produces commitments, challenges and final layers (azk_batch_trace), not proof bytes");
    uint64_t pos = 0;
    for (size_t i = 0; i < e.cfg.size(); i++) {
      layout(pos + e.proof_len[i] <= cap, "proof buffer too small");
      AZK_CU(cudaMemcpyAsync(out + pos, e.h_inst[i].proof, e.proof_len[i], cudaMemcpyDeviceToHost, e.s));
      pos += e.proof_len[i];
    }
    sync_stream(e.s);
  });
}

azk_status azk_batch_trace(azk_batch* b, uint32_t i, uint8_t* cm, uint32_t* ch, uint32_t* fl, uint32_t* qp) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b && i < b->eng.cfg.size());
    std::lock_guard<std::mutex> lk(b->mu);
    b->eng.trace(i, cm, ch, fl, qp);
  });
}

azk_status azk_batch_set_profiling(azk_batch* b, int enabled) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b != nullptr);
    std::lock_guard<std::mutex> lk(b->mu);
    b->eng.prof = enabled != 0;
  });
}

azk_status azk_batch_profile(azk_batch* b, double* seconds4) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b && seconds4);
    std::lock_guard<std::mutex> lk(b->mu);
    sync_stream(b->eng.s);
    b->eng.profile(seconds4);
  });
}

azk_status azk_batch_work(azk_batch* b, uint64_t* tree_permutations, uint64_t* fft_bytes, uint64_t* fold_bytes, uint32_t* launches) {
  return guarded(b ? b->ctx : nullptr, [&] {
    layout(b != nullptr);
    if (tree_permutations) *tree_permutations = b->eng.tree_perms;
    if (fft_bytes) *fft_bytes = b->eng.fft_bytes;
    if (fold_bytes) *fold_bytes = b->eng.fold_bytes;
    if (launches) *launches = b->eng.launches;
  });
}

void azk_batch_destroy(azk_batch* b) { delete b; }

}  // extern "C"

// ===========================================================================
// Continuous-batching server
//
// Jobs (Circle PCS commit-and-fold proofs and M31 multilinear sum-checks) enter
// one FIFO queue.  `slots` worker threads each own a CUDA stream; a worker takes
// the next queued job as soon as its device memory fits the HBM budget, so jobs
// that arrive while others run join the device as slots and memory free up and
// their kernels overlap with the running ones.
//
// Device memory is per worker and per job shape (a PCS engine or a sum-check
// table set), kept after the job for the next job of that shape: no allocation
// or free (each of which waits for the whole device) sits between jobs once the
// shapes have been seen.  Every byte held, in use or cached, counts against the
// budget; a worker whose next job does not fit first gives back its own cached
// shapes, least recently used first.
// ===========================================================================
namespace {

struct ServeJob {
  uint64_t id = 0;
  int kind = 0;  // 0 pcs, 1 sumcheck
  uint32_t logn = 0, rounds = 0, queries = 0, log_blowup = 0;
  std::vector<uint32_t> input;  // pcs: coefficient words; sumcheck: evaluations
  uint64_t count = 0;           // pcs: coefficient count
  bool zeros = false;           // warm-up job: `count` zero coefficients, no `input`
  uint8_t pub[32] = {0};
  uint64_t bytes = 0;  // device memory of its shape
  std::chrono::steady_clock::time_point submitted, started, finished;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  std::string error;
  std::vector<uint8_t> result;
};

using ShapeKey = std::tuple<int, uint32_t, uint32_t, uint32_t, uint32_t>;

ShapeKey shape_of(const ServeJob& j) { return std::make_tuple(j.kind, j.logn, j.rounds, j.queries, j.log_blowup); }

struct SumcheckBufs {
  DevBuf ev, scratch, rounds, out;
};

// Device memory of one job shape held by a worker.
struct Resident {
  std::unique_ptr<Engine> eng;
  std::unique_ptr<SumcheckBufs> sc;
  uint64_t bytes = 0;
  uint64_t last_use = 0;
};

uint64_t pcs_shape_bytes(uint32_t logn, uint32_t rounds, uint32_t queries) {
  uint64_t N = 1ull << logn;
  // arena of one engine: input 16N, layers 32N, trees 64N, tree counters 2N,
  // transcript and proof state; FFT work lists and slack rounded into 8N
  return 120 * N + proof_total_bytes(logn, rounds, queries, 0, false) + (64ull << 10);
}

uint64_t sumcheck_shape_bytes(uint32_t logn) { return 8ull << logn | 4096; }

}  // namespace

struct azk_server {
  azk_ctx* ctx;
  Sched sched;
  uint64_t budget;
  uint32_t slots;
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<std::shared_ptr<ServeJob>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<ServeJob>> jobs;
  uint64_t next_id = 1;
  uint64_t held = 0;  // device bytes held by all workers (in use and cached)
  uint64_t running = 0;
  uint64_t tick = 0;
  bool stop = false;
  std::vector<std::map<ShapeKey, Resident>> cache;  // per worker
  std::vector<uint8_t> busy;                         // per worker: running a job (its cache must stay)
  // per worker: jobs of zeros it runs once before serving (azk_server_warm), so its
  // engines, sum-check buffers and pinned staging exist before the first real job
  std::vector<std::deque<std::shared_ptr<ServeJob>>> warm;
  uint64_t warm_pending = 0;
  std::vector<cudaStream_t> streams;  // one per worker
  std::vector<std::thread> workers;
  uint64_t completed = 0, elems = 0;
  std::chrono::steady_clock::time_point first_submit, last_finish;
  bool any_submit = false;
};

namespace {

// Page-locked host staging of one worker: job inputs and results cross PCIe from
// here (copies from pageable memory go through the driver's own staging, which
// serialises the workers' copies).
struct Staging {
  uint8_t* p = nullptr;
  size_t n = 0;
  uint8_t* ensure(size_t bytes) {
    if (bytes > n) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      n = 0;
      size_t want = std::max<size_t>(bytes, 1 << 20);
      AZK_CU(cudaHostAlloc(reinterpret_cast<void**>(&p), want, cudaHostAllocDefault));
      n = want;
    }
    return p;
  }
  ~Staging() {
    if (p) cudaFreeHost(p);
  }
};

void run_pcs(azk_server* sv, Resident& r, ServeJob& j, Staging& st, cudaStream_t s) {
  if (!r.eng) {
    r.eng = std::make_unique<Engine>();
    Sched sc = sv->sched;
    sc.graph = false;
    r.eng->init(sv->ctx, {InstanceCfg{j.logn, j.rounds, j.queries, j.log_blowup, 0, {}}}, sc, s, s);
  }
  Engine* e = r.eng.get();
  const uint64_t in_bytes = 16 * j.count, proof = e->proof_len[0];
  uint8_t* pin = st.ensure(std::max<uint64_t>(in_bytes, proof) + 64);
  if (j.zeros)
    std::memset(pin, 0, in_bytes);
  else
    std::memcpy(pin, j.input.data(), in_bytes);
  uint4* in = e->arena.at<uint4>(e->off_input[0]);
  AZK_CU(cudaMemcpyAsync(in, pin, in_bytes, cudaMemcpyHostToDevice, e->s_up));
  e->scan_inputs({j.count});
  e->set_publics(j.pub);
  Timer t;
  e->run(true, true, nullptr, t);
  AZK_CU(cudaMemcpyAsync(pin, e->h_inst[0].proof, proof, cudaMemcpyDeviceToHost, e->s));
  sync_stream(e->s);
  j.result.assign(pin, pin + proof);
}

// Sum-check of one table through reusable device buffers: evaluations upload,
// one single-CTA kernel, results download.  Output words: claimed sum, final
// evaluation, digest (8 words), sums at 0, sums at 1, challenges (rounds each).
// `evals` and `pin` (>= 4n + sizeof(SumcheckOut) + 12 log n bytes) may be the same
// page-locked buffer: the evaluations are consumed by the upload before the
// results land.
std::vector<uint32_t> sumcheck_run(SumcheckBufs& b, const uint32_t* evals, uint32_t logn, cudaStream_t s, uint8_t* pin, double* gpu_s = nullptr) {
  const uint64_t n = 1ull << logn;
  if (!b.ev.p) {
    b.ev.alloc(4 * n, "Sumcheck.Evals");
    b.scratch.alloc(4 * n, "Sumcheck.Scratch");
    b.rounds.alloc(12ull * logn + 64, "Sumcheck.Rounds");
    b.out.alloc(sizeof(SumcheckOut), "Sumcheck.Out");
  }
  AZK_CU(cudaMemcpyAsync(b.ev.p, evals, 4 * n, cudaMemcpyHostToDevice, s));
  SumcheckOut* h = reinterpret_cast<SumcheckOut*>(pin + align_up(4 * n, 64));
  uint32_t* rounds_h = reinterpret_cast<uint32_t*>(h + 1);
  SumcheckOut ptrs{};
  ptrs.r0 = b.rounds.as<uint32_t>();
  ptrs.r1 = ptrs.r0 + logn;
  ptrs.challenges = ptrs.r1 + logn;
  *h = ptrs;
  AZK_CU(cudaMemcpyAsync(b.out.p, h, sizeof(SumcheckOut), cudaMemcpyHostToDevice, s));
  std::unique_ptr<GpuTimer> gt;
  if (gpu_s) gt.reset(new GpuTimer(s));  // the two kernels, digest and rounds
  AZK_CU(launch_sumcheck(b.ev.as<uint32_t>(), logn, b.scratch.as<uint32_t>(), b.out.as<SumcheckOut>(), s));
  if (gt) gt->stop();
  AZK_CU(cudaMemcpyAsync(h, b.out.p, sizeof(SumcheckOut), cudaMemcpyDeviceToHost, s));
  AZK_CU(cudaMemcpyAsync(rounds_h, b.rounds.p, 12ull * logn, cudaMemcpyDeviceToHost, s));
  sync_stream(s);
  if (gt) *gpu_s = gt->seconds();
  const SumcheckOut r = *h;
  std::vector<uint32_t> rounds(rounds_h, rounds_h + 3 * logn);
  std::vector<uint32_t> words = {r.claimed_sum, r.final_eval};
  for (int i = 0; i < 4; i++) {
    words.push_back((uint32_t)r.digest[i]);
    words.push_back((uint32_t)(r.digest[i] >> 32));
  }
  words.insert(words.end(), rounds.begin(), rounds.end());
  return words;
}

uint64_t sumcheck_pinned_bytes(uint32_t logn) { return align_up(4ull << logn, 64) + sizeof(SumcheckOut) + 12ull * logn + 64; }

void run_sumcheck(Resident& res, cudaStream_t s, ServeJob& j, Staging& st) {
  if (!res.sc) res.sc = std::make_unique<SumcheckBufs>();
  uint8_t* pin = st.ensure(sumcheck_pinned_bytes(j.logn));
  std::memcpy(pin, j.input.data(), 4ull << j.logn);
  std::vector<uint32_t> words = sumcheck_run(*res.sc, reinterpret_cast<const uint32_t*>(pin), j.logn, s, pin);
  j.result.resize(4 * words.size());
  std::memcpy(j.result.data(), words.data(), j.result.size());
}

// Evict the least recently used cached shape of worker `w` into `dropped` (its
// device memory is freed by the caller after the server lock is released: a free
// waits for the whole device).  Returns false when the worker caches nothing.
bool evict_lru(azk_server* sv, int w, std::vector<Resident>& dropped) {
  auto& cache = sv->cache[w];
  if (cache.empty()) return false;
  auto lru = cache.begin();
  for (auto it = cache.begin(); it != cache.end(); ++it)
    if (it->second.last_use < lru->second.last_use) lru = it;
  sv->held -= lru->second.bytes;
  dropped.push_back(std::move(lru->second));
  cache.erase(lru);
  return true;
}

// Called with the server lock held.  Takes the front job if its shape is cached
// by this worker or its bytes fit the budget.  To make room it evicts this
// worker's least recently used shapes first, then those of idle workers (a worker
// that is not running a job has nothing in flight on its stream, so its cached
// memory can go); busy workers keep theirs.  Nothing is taken while the job cannot
// fit; a job larger than the budget never enters the queue.  Evicted memory is
// handed back in `dropped` for the caller to free outside the lock.
std::shared_ptr<ServeJob> try_take(azk_server* sv, int w, std::vector<Resident>& dropped) {
  // this worker's warm-up jobs first; one that cannot fit the budget is dropped
  while (!sv->warm[w].empty()) {
    auto j = sv->warm[w].front();
    auto& cache = sv->cache[w];
    ShapeKey key = shape_of(*j);
    if (!cache.count(key)) {
      if (sv->held + j->bytes > sv->budget) {
        sv->warm[w].pop_front();
        sv->warm_pending--;
        sv->done_cv.notify_all();
        continue;
      }
      Resident& r = cache[key];
      r.bytes = j->bytes;
      sv->held += j->bytes;
    }
    cache[key].last_use = ++sv->tick;
    sv->warm[w].pop_front();
    sv->busy[w] = 1;
    j->state = 1;
    return j;
  }
  if (sv->queue.empty()) return nullptr;
  auto& cache = sv->cache[w];
  const auto& j = sv->queue.front();
  ShapeKey key = shape_of(*j);
  if (!cache.count(key)) {
    while (sv->held + j->bytes > sv->budget && evict_lru(sv, w, dropped)) {
    }
    for (uint32_t v = 0; v < sv->slots && sv->held + j->bytes > sv->budget; v++) {
      if ((int)v == w || sv->busy[v]) continue;
      while (sv->held + j->bytes > sv->budget && evict_lru(sv, (int)v, dropped)) {
      }
    }
    if (sv->held + j->bytes > sv->budget) return nullptr;
    Resident& r = cache[key];
    r.bytes = j->bytes;
    sv->held += j->bytes;
  }
  cache[key].last_use = ++sv->tick;
  auto job = j;
  sv->queue.pop_front();
  sv->running++;
  sv->busy[w] = 1;
  job->state = 1;
  job->started = std::chrono::steady_clock::now();
  return job;
}

void worker_loop(azk_server* sv, int w) {
  cudaSetDevice(sv->ctx->device);
  // everything this worker runs (uploads, proof kernels, sum-checks) goes on its one
  // stream: its jobs run one at a time, and one stream per worker keeps each worker
  // on its own hardware work queue (see azk_server_create)
  cudaStream_t s = sv->streams[w];
  Staging staging;
  for (;;) {
    std::shared_ptr<ServeJob> job;
    Resident* res = nullptr;
    std::vector<Resident> dropped;  // evicted shapes, freed below without the lock
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      for (;;) {
        if (sv->stop && sv->queue.empty() && sv->warm[w].empty()) break;
        job = try_take(sv, w, dropped);
        if (job) break;
        if (!dropped.empty()) {  // free what was evicted, then look again
          lk.unlock();
          dropped.clear();
          lk.lock();
          continue;
        }
        sv->cv.wait(lk);
      }
      if (!job) break;
      res = &sv->cache[w][shape_of(*job)];
    }
    dropped.clear();
    // the outcome is published under the lock together with the finish time, so a
    // poll never sees a finished job without its latency
    int outcome = 2;
    std::string error;
    try {
      if (job->kind == 0)
        run_pcs(sv, *res, *job, staging, s);
      else
        run_sumcheck(*res, s, *job, staging);
    } catch (const Error& e) {
      error = e.msg;
      outcome = 3;
    } catch (const std::exception& e) {
      error = e.what();
      outcome = 3;
    }
    std::vector<Resident> failed;  // a failed job's shape, freed without the lock
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      job->error = error;
      job->state = outcome;
      sv->busy[w] = 0;
      if (job->id == 0) {  // a warm-up job: not a result anyone polls
        if (job->state == 3) {
          auto it = sv->cache[w].find(shape_of(*job));
          if (it != sv->cache[w].end()) {
            sv->held -= it->second.bytes;
            failed.push_back(std::move(it->second));
            sv->cache[w].erase(it);
          }
        }
        sv->warm_pending--;
        sv->cv.notify_all();
        sv->done_cv.notify_all();
      }
      if (job->id == 0) continue;
      job->finished = std::chrono::steady_clock::now();
      job->input.clear();
      job->input.shrink_to_fit();
      if (job->state == 3) {  // drop the shape's memory: it may be in an unknown state
        auto it = sv->cache[w].find(shape_of(*job));
        if (it != sv->cache[w].end()) {
          sv->held -= it->second.bytes;
          failed.push_back(std::move(it->second));
          sv->cache[w].erase(it);
        }
      }
      sv->running--;
      sv->completed++;
      if (job->kind == 0 && job->state == 2) sv->elems += 1ull << job->logn;
      sv->last_finish = job->finished;
    }
    sv->cv.notify_all();
    sv->done_cv.notify_all();
  }
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (auto& kv : sv->cache[w]) sv->held -= kv.second.bytes;
    sv->cache[w].clear();
  }
}

uint64_t submit(azk_server* sv, std::shared_ptr<ServeJob> j) {
  std::lock_guard<std::mutex> lk(sv->mu);
  require(j->bytes <= sv->budget, AZK_ERR_HBM_BUDGET,
          "job needs " + std::to_string(j->bytes) + " device bytes, more than the server's HBM budget of " + std::to_string(sv->budget));
  j->id = sv->next_id++;
  j->submitted = std::chrono::steady_clock::now();
  if (!sv->any_submit) {
    sv->first_submit = j->submitted;
    sv->any_submit = true;
  }
  sv->jobs[j->id] = j;
  sv->queue.push_back(j);
  sv->cv.notify_all();
  return j->id;
}

}  // namespace

extern "C" {

azk_status azk_sumcheck_prove(azk_ctx* ctx, const uint32_t* evals, uint64_t count, uint32_t* sums0, uint32_t* sums1, uint32_t* challenges,
                              uint32_t* claimed_sum, uint32_t* final_eval, uint8_t digest[32], azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && evals && sums0 && sums1 && challenges && claimed_sum && final_eval && digest);
    // preconditions of M31MultilinearSumcheckProofBuilderV1.prove (SumcheckOracle.swift:803-807)
    layout(count > 1 && is_pow2(count) && count <= (1ull << 28), "evaluation count must be a power of two greater than one");
    for (uint64_t i = 0; i < count; i++) layout(evals[i] < kP, "input contains a non-canonical field element");
    std::lock_guard<std::mutex> lk(ctx->mu);
    Timer t;
    uint32_t logn = ilog2(count);
    SumcheckBufs b;
    Staging staging;
    uint8_t* pin = staging.ensure(sumcheck_pinned_bytes(logn));
    std::memcpy(pin, evals, 4ull << logn);
    double gpu_s = 0.0;
    std::vector<uint32_t> w = sumcheck_run(b, reinterpret_cast<const uint32_t*>(pin), logn, ctx->stream, pin, &gpu_s);
    *claimed_sum = w[0];
    *final_eval = w[1];
    std::memcpy(digest, w.data() + 2, 32);
    std::memcpy(sums0, w.data() + 10, 4ull * logn);
    std::memcpy(sums1, w.data() + 10 + logn, 4ull * logn);
    std::memcpy(challenges, w.data() + 10 + 2 * logn, 4ull * logn);
    fill_stats(st, t, 0, gpu_s);
  });
}

azk_status azk_server_create(azk_ctx* ctx, uint64_t hbm_budget_bytes, uint32_t slots, const azk_schedule* schedule, azk_server** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && slots >= 1 && slots <= 64 && hbm_budget_bytes > 0);
    auto sv = std::make_unique<azk_server>();
    sv->ctx = ctx;
    // each job is one instance: the single-tree table (measured on the serving mix:
    // the lowest latency per job at a throughput equal to the batch table's within
    // run-to-run spread)
    sv->sched = resolve_schedule(schedule, kTuned_pcs_single);
    sv->budget = hbm_budget_bytes;
    sv->slots = slots;
    sv->cache.resize(slots);
    sv->warm.resize(slots);
    // The workers' streams are created here, one after another, so that with up to
    // CUDA_DEVICE_MAX_CONNECTIONS (32) workers each lands on its own hardware work
    // queue.  Streams that share a queue wait on each other's dependent launches:
    // a sum-check's 64 ms digest followed by its rounds kernel then stalls every
    // stream behind it (measured with two streams per cached engine, ~800 streams:
    // completions stopped for up to a second at a time).  Highest priority: a
    // sum-check digest or a job's input scan takes the first free SM slot.
    int prio_lo = 0, prio_hi = 0;
    AZK_CU(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    sv->streams.assign(slots, nullptr);
    for (uint32_t w = 0; w < slots; w++) AZK_CU(cudaStreamCreateWithPriority(&sv->streams[w], cudaStreamNonBlocking, prio_hi));
    for (uint32_t w = 0; w < slots; w++) sv->workers.emplace_back(worker_loop, sv.get(), (int)w);
    *out = sv.release();
  });
}

azk_status azk_server_submit_pcs(azk_server* sv, uint32_t logn, uint32_t log_blowup, uint32_t queries, uint32_t rounds, const uint32_t* coeffs,
                                 uint64_t count, const uint8_t pub[32], uint64_t* job_id) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv && coeffs && pub && job_id);
    validate_params(logn, log_blowup, queries, 0, rounds);
    layout(count >= 1 && count <= (1ull << logn));
    for (uint64_t i = 0; i < 4 * count; i++) layout(coeffs[i] < kP, "input contains a non-canonical field element");
    auto j = std::make_shared<ServeJob>();
    j->kind = 0;
    j->logn = logn;
    j->rounds = rounds;
    j->queries = queries;
    j->log_blowup = log_blowup;
    j->input.assign(coeffs, coeffs + 4 * count);
    j->count = count;
    std::memcpy(j->pub, pub, 32);
    j->bytes = pcs_shape_bytes(logn, rounds, queries);
    *job_id = submit(sv, j);
  });
}

azk_status azk_server_warm(azk_server* sv, const uint32_t* pcs_logn, const uint32_t* pcs_rounds, uint32_t n_pcs, uint32_t log_blowup,
                           uint32_t queries, const uint32_t* sumcheck_logn, uint32_t n_sumcheck) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv && (n_pcs == 0 || (pcs_logn && pcs_rounds)) && (n_sumcheck == 0 || sumcheck_logn));
    for (uint32_t i = 0; i < n_pcs; i++) validate_params(pcs_logn[i], log_blowup, queries, 0, pcs_rounds[i]);
    for (uint32_t i = 0; i < n_sumcheck; i++) layout(sumcheck_logn[i] >= 1 && sumcheck_logn[i] <= 28);
    std::unique_lock<std::mutex> lk(sv->mu);
    for (uint32_t w = 0; w < sv->slots; w++) {
      for (uint32_t i = 0; i < n_pcs; i++) {
        auto j = std::make_shared<ServeJob>();  // id 0: a warm-up job
        j->kind = 0;
        j->logn = pcs_logn[i];
        j->rounds = pcs_rounds[i];
        j->queries = queries;
        j->log_blowup = log_blowup;
        // all 2^logn coefficients (zeros): the worker's pinned staging grows to the
        // largest input of the shape now, not in the middle of serving, where
        // freeing the smaller buffer would wait for the whole device
        j->zeros = true;
        j->count = 1ull << j->logn;
        j->bytes = pcs_shape_bytes(j->logn, j->rounds, j->queries);
        sv->warm[w].push_back(j);
        sv->warm_pending++;
      }
      for (uint32_t i = 0; i < n_sumcheck; i++) {
        auto j = std::make_shared<ServeJob>();
        j->kind = 1;
        j->logn = sumcheck_logn[i];
        j->input.assign(1ull << j->logn, 0u);
        j->bytes = sumcheck_shape_bytes(j->logn);
        sv->warm[w].push_back(j);
        sv->warm_pending++;
      }
    }
    sv->cv.notify_all();
    sv->done_cv.wait(lk, [&] { return sv->warm_pending == 0; });
  });
}

azk_status azk_server_submit_sumcheck(azk_server* sv, const uint32_t* evals, uint64_t count, uint64_t* job_id) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv && evals && job_id);
    // M31MultilinearSumcheckProofBuilderV1.prove preconditions (SumcheckOracle.swift:803-807)
    layout(count > 1 && is_pow2(count) && count <= (1ull << 28));
    for (uint64_t i = 0; i < count; i++) layout(evals[i] < kP, "input contains a non-canonical field element");
    auto j = std::make_shared<ServeJob>();
    j->kind = 1;
    j->logn = ilog2(count);
    j->input.assign(evals, evals + count);
    j->bytes = sumcheck_shape_bytes(j->logn);
    *job_id = submit(sv, j);
  });
}

azk_status azk_server_poll(azk_server* sv, uint64_t id, int* state, double* latency_s, uint8_t* out, uint64_t* out_len) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv && state);
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    layout(it != sv->jobs.end(), "unknown job id");
    ServeJob& j = *it->second;
    *state = j.state;
    if (j.state == 3) fail(AZK_ERR_COMMAND_EXECUTION_FAILED, j.error);
    if (j.state == 2) {
      if (latency_s) *latency_s = std::chrono::duration<double>(j.finished - j.submitted).count();
      if (out_len) {
        if (out) {
          layout(*out_len >= j.result.size(), "result buffer too small");
          std::memcpy(out, j.result.data(), j.result.size());
        }
        *out_len = j.result.size();
      }
    }
  });
}

azk_status azk_server_release(azk_server* sv, uint64_t id) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv != nullptr);
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->jobs.find(id);
    layout(it != sv->jobs.end() && it->second->state >= 2, "job not finished");
    sv->jobs.erase(it);
  });
}

azk_status azk_server_wait_all(azk_server* sv) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv != nullptr);
    std::unique_lock<std::mutex> lk(sv->mu);
    sv->done_cv.wait(lk, [&] { return sv->queue.empty() && sv->running == 0; });
  });
}

azk_status azk_server_stats(azk_server* sv, uint64_t* completed, uint64_t* elems, double* span_s, uint64_t* held) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv != nullptr);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (completed) *completed = sv->completed;
    if (elems) *elems = sv->elems;
    if (span_s) *span_s = sv->any_submit ? std::chrono::duration<double>(sv->last_finish - sv->first_submit).count() : 0.0;
    if (held) *held = sv->held;
  });
}

void azk_server_destroy(azk_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv.notify_all();
  for (auto& t : sv->workers) t.join();
  for (auto st : sv->streams)
    if (st) cudaStreamDestroy(st);
  delete sv;
}

}  // extern "C"
