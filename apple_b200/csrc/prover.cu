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
#include <map>
#include <memory>
#include <algorithm>
#include <condition_variable>
#include <deque>
#include <set>
#include <thread>
#include <tuple>
#include <unordered_map>

#include "azk_field.cuh"
#include "azk_runtime.h"
#include "azk_tuned.h"

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
  uint64_t off_inst = 0, off_flag = 0, off_info = 0, off_queue = 0;  // off_queue: two words per round (persistent trees)

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
  std::vector<uint32_t> tstep_log;                                      // largest layer log per step
  std::vector<FoldJob> fold_jobs;
  std::vector<uint2> fold_work;
  std::vector<uint64_t> fstep_off, fstep_cnt;
  std::vector<std::vector<std::pair<uint64_t, uint64_t>>> fstep_inst;
  std::vector<uint32_t> ids;
  DevBuf d_tree_jobs, d_tree_work, d_fold_jobs, d_fold_work, d_ids;

  // Captured launch sequences, keyed by the FFT work-list set in use (its narrow
  // flags), the input kind and the active-instance count (0: all).  Every FFT
  // work-list set keeps its own device lists (`fft` in use, `fft_saved` the
  // others), so a graph stays valid while other sets run.
  using GraphKey = std::tuple<std::vector<uint8_t>, bool, uint32_t>;
  std::map<GraphKey, cudaGraphExec_t> graphs;
  std::map<std::vector<uint8_t>, FftPlan> fft_saved;
  static constexpr size_t kMaxGraphs = 64, kMaxFftSets = 16;
  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.second);
    graphs.clear();
  }

  // Kept for the engine's lifetime, so a run creates and destroys nothing: the
  // run's timing events, and page-locked words for the input scan's readbacks
  // (two status words at 0 and 16, then the per-instance input descriptions and
  // the scan's job list).
  cudaEvent_t tm_a = nullptr, tm_b = nullptr;
  HostPinned hsmall;
  uint32_t* hword(int k) const { return reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(hsmall.p) + 16 * k); }
  InputInfo* hinfo() const { return reinterpret_cast<InputInfo*>(static_cast<uint8_t*>(hsmall.p) + 64); }
  ScanJob* hscan() const {
    return reinterpret_cast<ScanJob*>(static_cast<uint8_t*>(hsmall.p) + 64 + align_up(sizeof(InputInfo) * cfg.size(), 16));
  }

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
    drop_graphs();
    for (auto e : ev_a) cudaEventDestroy(e);
    for (auto e : ev_b) cudaEventDestroy(e);
    if (tm_a) cudaEventDestroy(tm_a);
    if (tm_b) cudaEventDestroy(tm_b);
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
  // `counts` covers the first counts.size() instances (a server group runs a prefix
  // of its engine's instances).
  void scan_inputs(const std::vector<uint64_t>& counts) {
    const size_t m = counts.size();
    InputInfo* h = hinfo();
    ScanJob* jobs = hscan();
    uint32_t* f = hword(0);
    for (size_t i = 0; i < m; i++) h[i] = InputInfo{1u, 0u, counts[i]};
    AZK_CU(cudaMemcpyAsync(d_info(), h, sizeof(InputInfo) * m, cudaMemcpyHostToDevice, s_up));
    AZK_CU(cudaMemsetAsync(d_flag(), 0, 4, s_up));
    uint64_t max_n = 0;
    for (size_t i = 0; i < m; i++) {
      const uint64_t N = 1ull << cfg[i].logn;
      jobs[i] = ScanJob{arena.at<uint4>(off_input[i]), counts[i], N, d_info() + i};
      max_n = std::max(max_n, N);
    }
    if (!d_scan.p) d_scan.alloc(sizeof(ScanJob) * cfg.size(), "PCS.ScanJobs");
    AZK_CU(cudaMemcpyAsync(d_scan.p, jobs, sizeof(ScanJob) * m, cudaMemcpyHostToDevice, s_up));
    AZK_CU(launch_scan_inputs(d_scan.as<ScanJob>(), (uint32_t)m, max_n, d_flag(), s_up));
    AZK_CU(cudaMemcpyAsync(f, d_flag(), 4, cudaMemcpyDeviceToHost, s_up));
    AZK_CU(cudaMemcpyAsync(h, d_info(), sizeof(InputInfo) * m, cudaMemcpyDeviceToHost, s_up));
    sync_stream(s_up);
    layout(*f == 0, "input contains a non-canonical field element");
    std::vector<uint8_t> narrow(m);
    for (size_t i = 0; i < m; i++) narrow[i] = h[i].m31 ? 1 : 0;
    set_fft_narrow(narrow);
  }
  // Inputs written by the caller through a device pointer: nothing known.
  void forget_input(size_t i) {
    AZK_CU(cudaMemsetAsync(d_info() + i, 0, sizeof(InputInfo), s));
    std::vector<uint8_t> narrow = fft_narrow;
    narrow[i] = 0;
    set_fft_narrow(narrow);
  }
  // Which instances run the one-limb FFT kernel; `narrow` covers the transforms of
  // the first narrow.size() instances (the FFT runs over those).  A set of flags
  // seen before gets its saved work lists back (and its graphs stay valid); a new
  // one builds lists of its own.  Past kMaxFftSets saved sets, the saved sets and
  // every graph are dropped.
  void set_fft_narrow(const std::vector<uint8_t>& narrow) {
    if (narrow == fft_narrow) return;
    sync_stream(s);
    auto it = fft_saved.find(narrow);
    FftPlan next;
    const bool saved = it != fft_saved.end();
    if (saved) {
      next = std::move(it->second);
      fft_saved.erase(it);
    }
    fft_saved[fft_narrow] = std::move(fft);
    if (saved) {
      fft = std::move(next);
    } else {
      fft = FftPlan();
      fft.build(std::vector<FftJob>(fft_transforms.begin(), fft_transforms.begin() + narrow.size()), narrow);
      fft.upload(s);
      sync_stream(s);
    }
    fft_narrow = narrow;
    if (fft_saved.size() > kMaxFftSets) {
      drop_graphs();
      fft_saved.clear();
    }
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
    if (!tm_a) AZK_CU(cudaEventCreate(&tm_a));
    if (!tm_b) AZK_CU(cudaEventCreate(&tm_b));
    hsmall.ensure(64 + align_up(sizeof(InputInfo) * n, 16) + sizeof(ScanJob) * n);
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
    off_queue = arena.reserve(8ull * (rmax + 1));
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
    tstep_log.assign(rmax, 0);
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
        tstep_log[k] = std::max(tstep_log[k], lg);
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
    for (auto& st : fft.part_cnt)
      for (auto c3 : st) launches += c3 ? 1 : 0;
    for (auto c3 : tstep_cnt) launches += c3 ? 1 : 0;
    for (auto c3 : fstep_cnt) launches += c3 ? 1 : 0;
    launches += 4;  // prefix, finalize, queries, emit
    ensure_events(fft.steps() + 2 * rmax + 8);
  }

  uint32_t tree_kind(uint32_t k) const {
    if (leaf_values == 4) return k == 0 ? kLeafQM31x4 : kLeafFoldx4;
    return k == 0 ? kLeafQM31 : kLeafFold;
  }
  // `lg`: the largest layer (log leaves) the launch commits; its threads per CTA
  void launch_tree_range(uint32_t k, uint64_t off, uint64_t cnt, uint32_t lg) {
    if (!cnt) return;
    AZK_CU(launch_tree_jobs(d_tree_jobs.as<TreeJob>(), d_tree_work.as<uint2>() + off, (uint32_t)cnt, tstep_tile[k], tree_kind(k),
                            tree_threads(sched, lg), s, sched.persistent_trees ? arena.at<uint32_t>(off_queue) + 2 * k : nullptr));
  }
  uint32_t layer_log(uint32_t i, uint32_t k) const { return cfg[i].logn - k - (leaf_values == 4 ? 2 : 0); }
  void launch_fold_range(uint64_t off, uint64_t cnt) {
    if (!cnt) return;
    AZK_CU(launch_fold_jobs(d_fold_jobs.as<FoldJob>(), d_fold_work.as<uint2>() + off, (uint32_t)cnt, s));
  }

  // Instances a batched run covers: all of them, or the first n_act of an engine
  // whose instances all have one shape (a server group; its work lists are then
  // instance-major, so the first n_act instances' items are a prefix of every step).
  uint32_t n_act = 0;
  uint32_t active() const { return n_act ? n_act : (uint32_t)cfg.size(); }
  uint64_t tree_step_count(uint32_t k) const {
    if (!n_act) return tstep_cnt[k];
    uint64_t c = 0;
    for (uint32_t i = 0; i < n_act; i++) c += tstep_inst[k][i].second;
    return c;
  }
  uint64_t fold_step_count(uint32_t k) const {
    if (!n_act) return fstep_cnt[k];
    uint64_t c = 0;
    for (uint32_t i = 0; i < n_act; i++) c += fstep_inst[k][i].second;
    return c;
  }
  // Everything up to (not including) grinding.  from_coeffs: run the FFT first.
  void enqueue_rounds_batched(bool from_coeffs) {
    ev_used = 0;
    const uint32_t na = active();
    if (from_coeffs) {
      for (size_t st = 0; st < fft.steps(); st++) {
        prof_begin(0);
        fft.launch_step(st, s);
        prof_end();
      }
    }
    prof_begin(3);
    AZK_CU(launch_pcs_prefix(d_inst(), na, s));
    prof_end();
    for (uint32_t k = 0; k <= rmax; k++) {
      if (k < rmax) {
        prof_begin(1);
        launch_tree_range(k, tstep_off[k], tree_step_count(k), n_act ? layer_log(0, k) : tstep_log[k]);
        prof_end();
      }
      if (k >= 1 && fold_step_count(k)) {
        prof_begin(2);
        launch_fold_range(fstep_off[k], fold_step_count(k));
        prof_end();
      }
    }
    prof_begin(3);
    AZK_CU(launch_pcs_finalize(d_inst(), d_ids.as<uint32_t>(), na, s));
    prof_end();
  }
  // Proof bytes exist only for 16-byte leaves (the reference's verifier opens one
  // QM31 value per leaf); a 64-byte-leaf chain ends with its final layer.
  bool has_proofs() const { return leaf_values == 1; }
  void enqueue_tail_batched() {
    if (!has_proofs()) return;
    prof_begin(3);
    AZK_CU(launch_pcs_queries(d_inst(), d_ids.as<uint32_t>(), active(), s));
    AZK_CU(launch_pcs_emit(d_inst(), d_ids.as<uint32_t>(), active(), qmax, s));
    prof_end();
  }
  void enqueue_instance(uint32_t i, bool from_coeffs) {
    if (from_coeffs)
      for (size_t st = 0; st < fft.steps(); st++)
        if (fft.inst_range[st][i].second) fft.launch_step_for(st, i, s);
    AZK_CU(launch_pcs_prefix(d_inst() + i, 1, s));
    const uint32_t* id = d_ids.as<uint32_t>() + i;
    for (uint32_t k = 0; k <= cfg[i].rounds; k++) {
      if (k < cfg[i].rounds) launch_tree_range(k, tstep_inst[k][i].first, tstep_inst[k][i].second, layer_log(i, k));
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
    const size_t na = active();
    for (size_t i = 0; i < na; i++) std::memcpy(h_inst[i].pub, pubs + 32 * i, 32);
    AZK_CU(cudaMemcpy2DAsync(reinterpret_cast<uint8_t*>(d_inst()) + offsetof(PcsInstance, pub), sizeof(PcsInstance), pubs, 32, 32, na,
                             cudaMemcpyHostToDevice, s));
  }

  // Run the whole superstep; returns device seconds.
  double run(bool from_coeffs, bool plain, uint64_t* submit_ns, const Timer& t) {
    AZK_CU(cudaMemsetAsync(d_flag(), 0, 4, s));
    GpuTimer g(s, tm_a, tm_b);
    if (plain) {
      ev_used = 0;
      for (uint32_t i = 0; i < active(); i++) enqueue_instance(i, from_coeffs);
    } else if (!any_grinding && sched.graph && !prof) {
      // (profiled runs take the eager path below: the same launch sequence, with
      // event pairs around each stage)
      GraphKey key{fft_narrow, from_coeffs, n_act};
      auto it = graphs.find(key);
      if (it == graphs.end()) {
        if (graphs.size() >= kMaxGraphs) drop_graphs();
        cudaGraph_t gr;
        cudaGraphExec_t exec = nullptr;
        AZK_CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        enqueue_rounds_batched(from_coeffs);
        enqueue_tail_batched();
        AZK_CU(cudaStreamEndCapture(s, &gr));
        const cudaError_t e = cudaGraphInstantiate(&exec, gr, 0);
        cudaGraphDestroy(gr);
        AZK_CU(e);
        it = graphs.emplace(std::move(key), exec).first;
      }
      AZK_CU(cudaGraphLaunch(it->second, s));
    } else {
      enqueue_rounds_batched(from_coeffs);
      for (uint32_t i = 0; i < active(); i++) grind_instance(i);
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
    uint32_t* f = hword(1);
    AZK_CU(cudaMemcpyAsync(f, d_flag(), 4, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
    layout(*f == 0, "input contains a non-canonical field element");
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
  // monomial columns -> FFT basis on the device (made on first use)
  azk_witness_plan* wit = nullptr;
  DevBuf wx, wy;  // staging for host columns
  ~azk_pcs_prover() {
    if (wit) azk_witness_plan_destroy(wit);
  }
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
    Sched sc = resolve_schedule(schedule, kTuned_pcs_single, kTunedThreads_pcs_single);
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
  if (coeffs) e.fft.check_status(e.s);
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
    AZK_CU(cudaSetDevice(p->ctx->device));
    require_device_range(din, in_off, 16 * N);
    Timer t;
    pcs_ensure_claimed(p, {});
    require_device_range(dproof, 0, std::min<uint64_t>(*proof_len, p->eng.proof_len[0]));
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

}  // extern "C"

// Monomial coefficient columns (device) -> interleaved FFT-basis coefficients in
// the engine's input, through the witness plan's kernels (the conversion the
// reference's prove(polynomial:) runs on the CPU, CircleCodeword.swift:983-1005,
// and proveResidentWitnessCoefficients on the GPU, :1061-1080, 1235-1280); then the
// input scan over all N values (the line-basis step can spread nonzeros over the
// whole coefficient range).
static void pcs_witness_input(azk_pcs_prover* p, const void* dx, uint64_t x_off, uint64_t nx, const void* dy, uint64_t y_off, uint64_t ny) {
  if (!p->wit) {
    const azk_status s = azk_witness_plan_create(p->ctx, p->logn, &p->wit);
    if (s != AZK_OK) fail(s, azk_last_error_message(p->ctx));
  }
  Engine& e = p->eng;
  azk_stats ws{};
  const azk_status s = azk_witness_plan_execute_resident(p->wit, dx, x_off, nx, dy, y_off, ny, e.arena.buf.p, e.off_input[0], &ws);
  if (s != AZK_OK) fail(s, azk_last_error_message(p->ctx));
  e.scan_inputs({1ull << p->logn});
}

extern "C" {

azk_status azk_pcs_prover_prove_polynomial(azk_pcs_prover* p, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny, const uint8_t pub[32],
                                           uint8_t* proof_out, uint64_t* proof_len, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && pub && proof_out && proof_len && (x || !nx) && (y || !ny));
    const uint64_t half = (1ull << p->logn) / 2;
    layout(nx <= half && ny <= half, "each coefficient column holds at most half the domain size");
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    pcs_ensure_claimed(p, {});
    if (!p->wx.p) {
      p->wx.alloc(16 * std::max<uint64_t>(half, 1), "CirclePCSProver.WitnessX");
      p->wy.alloc(16 * std::max<uint64_t>(half, 1), "CirclePCSProver.WitnessY");
    }
    Engine& e = p->eng;
    if (nx) AZK_CU(cudaMemcpyAsync(p->wx.p, x, 16 * nx, cudaMemcpyHostToDevice, e.s));
    if (ny) AZK_CU(cudaMemcpyAsync(p->wy.p, y, 16 * ny, cudaMemcpyHostToDevice, e.s));
    sync_stream(e.s);
    pcs_witness_input(p, p->wx.p, 0, nx, p->wy.p, 0, ny);
    pcs_prove_common(p, true, pub, proof_out, false, proof_len, st, t);
  });
}

azk_status azk_pcs_prover_prove_resident_witness(azk_pcs_prover* p, const void* dev_x, uint64_t x_offset, uint64_t nx, const void* dev_y,
                                                 uint64_t y_offset, uint64_t ny, const uint8_t pub[32], void* dproof, uint64_t* proof_len,
                                                 azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && pub && dproof && proof_len);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    pcs_ensure_claimed(p, {});
    require_device_range(dproof, 0, std::min<uint64_t>(*proof_len, p->eng.proof_len[0]));
    pcs_witness_input(p, dev_x, x_offset, nx, dev_y, y_offset, ny);
    pcs_prove_common(p, true, pub, static_cast<uint8_t*>(dproof), true, proof_len, st, t);
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
    Sched sc = resolve_schedule(nullptr, kTuned_pcs_single, kTunedThreads_pcs_single);
    sc.graph = false;
    e.init(ctx, {InstanceCfg{logn, rounds, queries, log_blowup, grinding, {}}}, sc);
    AZK_CU(cudaMemcpyAsync(e.h_inst[0].layers, ev, 16 * N, cudaMemcpyHostToDevice, e.s));
    e.check_input_canonical(e.h_inst[0].layers, 4 * N);
    e.set_publics(pub);
    GpuTimer g(e.s);
    AZK_CU(launch_pcs_prefix(e.d_inst(), 1, e.s));
    for (uint32_t k = 0; k <= rounds; k++) {
      if (k < rounds) e.launch_tree_range(k, e.tstep_inst[k][0].first, e.tstep_inst[k][0].second, e.layer_log(0, k));
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
    b->eng.init(ctx, cf, resolve_schedule(schedule, kTuned_pcs_batch, kTunedThreads_pcs_batch));
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
    e.fft.check_status(e.s);
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
// one FIFO queue.  `slots` worker threads each own a CUDA stream.  A worker takes
// the front job as soon as its device memory fits the HBM budget, so jobs that
// arrive while others run join the device as slots and memory free up and their
// kernels overlap with the running ones:
//  - a PCS job is taken together with the other queued PCS jobs of its shape (up
//    to the shape's group capacity), and the group is proved as one batched
//    superstep on the worker's engine for that shape (one launch per stage over
//    the group's instances);
//  - a sum-check job is handed to the sum-check lane and the worker moves on: the
//    lane proves the tables that are waiting in one batched launch (one CTA per
//    table) on a few streams of its own, and a completion thread publishes each
//    batch's results when its event fires, so a 2^20 table's tens of milliseconds
//    of sequential digest never hold a worker.
//
// Device memory is per worker and per PCS shape (an engine with room for the
// shape's group capacity), plus the lane's table slots and the context's domain
// tables for each log size in use, all kept for later jobs: no allocation or free
// (each of which waits for the whole device) sits between jobs once the shapes
// have been seen.  Every byte held counts against the budget; to admit a job that
// does not fit, the taking worker gives back its own least recently used shapes,
// then those of idle workers.
// ===========================================================================
namespace {

struct ServeJob {
  uint64_t id = 0;
  int kind = 0;  // 0 pcs, 1 sumcheck
  uint32_t logn = 0, rounds = 0, queries = 0, log_blowup = 0;
  std::vector<uint32_t> input;        // pcs: coefficient words; sumcheck: evaluations
  const uint32_t* borrowed = nullptr;  // the caller's words instead of `input` (no-copy submission)
  uint64_t count = 0;                 // pcs: coefficient count
  bool zeros = false;                 // warm-up job: `count` zero coefficients, no `input`
  uint32_t warm_group = 1;            // warm-up job: proved as a group of this many copies
  uint8_t pub[32] = {0};
  std::chrono::steady_clock::time_point submitted, started, finished;
  int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
  std::string error;
  std::vector<uint8_t> result;
};

using ShapeKey = std::tuple<uint32_t, uint32_t, uint32_t, uint32_t>;  // PCS: logn, rounds, queries, log_blowup

ShapeKey shape_of(const ServeJob& j) { return std::make_tuple(j.logn, j.rounds, j.queries, j.log_blowup); }

const uint32_t* job_words(const ServeJob& j) { return j.borrowed ? j.borrowed : j.input.data(); }
// Once a job's words are in page-locked staging nothing reads them again: its copy
// goes back to the allocator (so the next submission reuses warm pages) and a
// borrowed pointer is forgotten.  Only the thread that holds the job calls this.
void drop_input(ServeJob& j) {
  std::vector<uint32_t>().swap(j.input);
  j.borrowed = nullptr;
}

// Jobs of one shape proved together, at most: 8 up to 2^17 values, then halving
// (4 at 2^18, 2 at 2^19), one from 2^20 on, where one job already fills the GPU's
// launches.
uint32_t group_capacity(uint32_t logn) { return logn >= 20 ? 1u : logn >= 17 ? (1u << (20 - logn)) : 8u; }

// Device bytes of one PCS instance: input 16N, layers 32N, trees 64N, tree
// counters, transcript, proof; work lists and slack rounded into 8N.
uint64_t pcs_instance_bytes(uint32_t logn, uint32_t rounds, uint32_t queries) {
  const uint64_t N = 1ull << logn;
  return 120 * N + proof_total_bytes(logn, rounds, queries, 0, false) + 4096;
}
uint64_t pcs_engine_bytes(uint32_t logn, uint32_t rounds, uint32_t queries, uint32_t cap) {
  return cap * pcs_instance_bytes(logn, rounds, queries) + (64ull << 10);
}
// Domain tables of a log size (FFT twiddles, their doubled copy and their
// inverses, N words each).
uint64_t domain_bytes(uint32_t logn) { return 12ull << logn; }

struct SumcheckBufs {
  DevBuf ev, scratch, rounds, out;
};
uint64_t sumcheck_table_bytes(uint32_t logn) { return (8ull << logn) + 12ull * logn + 4096; }
uint64_t sumcheck_pinned_bytes(uint32_t logn) { return align_up(4ull << logn, 64) + sizeof(SumcheckOut) + 12ull * logn + 64; }

// Device memory of one PCS shape held by a worker.
struct Resident {
  std::unique_ptr<Engine> eng;
  uint32_t cap = 1;
  uint64_t bytes = 0;
  uint64_t last_use = 0;
};

// Page-locked host staging: job inputs and results cross PCIe from here (copies
// from pageable memory go through the driver's own staging, which serialises the
// workers' copies).
struct Staging {
  uint8_t* p = nullptr;
  size_t n = 0;
  unsigned flags = cudaHostAllocDefault;
  uint8_t* ensure(size_t bytes) {
    if (bytes > n) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      n = 0;
      size_t want = std::max<size_t>(bytes, 1 << 20);
      AZK_CU(cudaHostAlloc(reinterpret_cast<void**>(&p), want, flags));
      n = want;
    }
    return p;
  }
  ~Staging() {
    if (p) cudaFreeHost(p);
  }
};

// One table slot of the sum-check lane: device buffers for a table of up to
// 2^cap_log words and page-locked, device-mapped staging for its input and
// results (the kernel writes the results straight into it).
struct SumcheckSlot {
  SumcheckBufs bufs;
  Staging pin;
  uint32_t cap_log = 0;  // 0: not allocated
  bool grow = false;     // cap_log was raised: the buffers are reallocated before use
  std::shared_ptr<ServeJob> job;
  SumcheckSlot() { pin.flags = cudaHostAllocMapped; }
};
// A lane stream and the batch it runs.  Nothing is queued on a lane stream after a
// batch's kernel (no event, no copy back): the completer polls the stream, so a
// worker stream that shares the lane stream's hardware queue never waits behind a
// queued operation that waits for the digest.
struct SumcheckStream {
  cudaStream_t s = nullptr;
  std::vector<int> slots;
};
constexpr int kLaneSlots = 256;  // tables in the lane at once (a packed CTA runs four, one per SM sub-partition)
constexpr int kLaneStreams = 32;               // batches in flight at once
constexpr int kLaneBatch = kSumcheckBatchMax;  // tables per launch

}  // namespace

struct azk_server {
  azk_ctx* ctx;
  Sched sched;
  uint64_t budget;
  uint32_t slots;
  std::mutex mu;
  std::condition_variable cv, done_cv, lane_cv;
  std::deque<std::shared_ptr<ServeJob>> queue;
  uint64_t queued_sc = 0;  // sum-check jobs in `queue`
  std::unordered_map<uint64_t, std::shared_ptr<ServeJob>> jobs;
  uint64_t next_id = 1;
  uint64_t held = 0;  // device bytes held (engines, lane slots, domain tables)
  uint64_t running = 0;
  uint64_t tick = 0;
  bool stop = false, lane_stop = false;
  std::vector<std::map<ShapeKey, Resident>> cache;  // per worker
  std::vector<uint8_t> busy;                         // per worker: running a job (its cache must stay)
  std::set<uint32_t> domain_logs;                    // log sizes whose domain tables are counted in `held`
  // per worker: jobs of zeros it runs once before serving (azk_server_warm), so its
  // engines and pinned staging exist before the first real job
  std::vector<std::deque<std::shared_ptr<ServeJob>>> warm;
  uint64_t warm_pending = 0;
  std::vector<cudaStream_t> streams;  // one per worker
  std::vector<std::thread> workers;
  // sum-check lane
  std::vector<std::unique_ptr<SumcheckSlot>> sc_slot;
  std::vector<int> sc_free;     // slots without a table
  std::deque<int> sc_pending;   // slots whose table waits for a launch
  std::vector<SumcheckStream> sc_stream;
  std::vector<int> sc_idle;     // lane streams without a batch
  std::deque<int> sc_inflight;  // lane streams with a batch, in launch order
  bool launcher_done = false;
  std::thread sc_launcher, sc_completer;
  uint64_t completed = 0, elems = 0, groups = 0, grouped = 0;
  std::chrono::steady_clock::time_point first_submit, last_finish;
  bool any_submit = false;
};

namespace {

// Group capacity of a shape under the server's budget: halved until the engine
// takes at most half the budget.
uint32_t shape_capacity(const azk_server* sv, const ServeJob& j) {
  uint32_t cap = group_capacity(j.logn);
  while (cap > 1 && pcs_engine_bytes(j.logn, j.rounds, j.queries, cap) > sv->budget / 2) cap >>= 1;
  return cap;
}

// Proves a group of same-shape PCS jobs on the worker's engine for the shape (made
// on first use with room for the shape's capacity): inputs staged and copied, one
// scan launch, one batched superstep over the group's instances (one CUDA graph
// launch: the engine captures the sequence once per group size), proofs read back.
void run_pcs_group(azk_server* sv, Resident& r, std::vector<std::shared_ptr<ServeJob>>& g, Staging& st, cudaStream_t s) {
  const ServeJob& j0 = *g[0];
  if (!r.eng) {
    r.eng = std::make_unique<Engine>();
    std::vector<InstanceCfg> cf(r.cap, InstanceCfg{j0.logn, j0.rounds, j0.queries, j0.log_blowup, 0, {}});
    r.eng->init(sv->ctx, cf, sv->sched, s, s);
  }
  Engine* e = r.eng.get();
  const size_t m = g.size();
  const uint64_t proof = e->proof_len[0];
  std::vector<uint64_t> off(m), counts(m);
  uint64_t in_total = 0;
  for (size_t i = 0; i < m; i++) {
    off[i] = in_total;
    counts[i] = g[i]->count;
    in_total += align_up(16 * g[i]->count, 64);
  }
  // warm-up jobs size the staging for a full group of complete inputs
  const uint64_t want = std::max<uint64_t>(std::max<uint64_t>(in_total, m * align_up(proof, 64)),
                                           j0.zeros ? r.cap * std::max<uint64_t>(16ull << j0.logn, align_up(proof, 64)) : 0);
  uint8_t* pin = st.ensure(want + 64);
  for (size_t i = 0; i < m; i++) {
    if (g[i]->zeros)
      std::memset(pin + off[i], 0, 16 * counts[i]);
    else
      std::memcpy(pin + off[i], job_words(*g[i]), 16 * counts[i]);
    drop_input(*g[i]);
    AZK_CU(cudaMemcpyAsync(e->arena.at<uint4>(e->off_input[i]), pin + off[i], 16 * counts[i], cudaMemcpyHostToDevice, e->s_up));
  }
  e->scan_inputs(counts);  // waits for the copies
  std::vector<uint8_t> pubs(32 * m);
  for (size_t i = 0; i < m; i++) std::memcpy(pubs.data() + 32 * i, g[i]->pub, 32);
  e->n_act = (uint32_t)m;
  e->set_publics(pubs.data());
  Timer t;
  e->run(true, false, nullptr, t);
  for (size_t i = 0; i < m; i++)
    AZK_CU(cudaMemcpyAsync(pin + i * align_up(proof, 64), e->h_inst[i].proof, proof, cudaMemcpyDeviceToHost, e->s));
  sync_stream(e->s);
  e->fft.check_status(e->s, e->hword(1));
  for (size_t i = 0; i < m; i++) g[i]->result.assign(pin + i * align_up(proof, 64), pin + i * align_up(proof, 64) + proof);
}

// Sum-check of one table through reusable device buffers (the single-table entry
// point): evaluations upload, one kernel, results download.  Output words: claimed
// sum, final evaluation, digest (8 words), sums at 0, sums at 1, challenges
// (rounds each).  `evals` and `pin` (>= sumcheck_pinned_bytes) may be the same
// page-locked buffer: the evaluations are consumed by the upload before the
// results land.
void sumcheck_alloc(SumcheckBufs& b, uint32_t logn) {
  const uint64_t n = 1ull << logn;
  b.ev.alloc(4 * n, "Sumcheck.Evals");
  b.scratch.alloc(4 * n, "Sumcheck.Scratch");
  b.rounds.alloc(12ull * logn + 64, "Sumcheck.Rounds");
  b.out.alloc(sizeof(SumcheckOut), "Sumcheck.Out");
}
// The SumcheckOut a table's kernel fills (per-round arrays in b.rounds).
SumcheckOut sumcheck_out_ptrs(const SumcheckBufs& b, uint32_t logn) {
  SumcheckOut o{};
  o.r0 = b.rounds.as<uint32_t>();
  o.r1 = o.r0 + logn;
  o.challenges = o.r1 + logn;
  return o;
}
std::vector<uint32_t> sumcheck_words(const SumcheckOut& r, const uint32_t* rounds_h, uint32_t logn) {
  std::vector<uint32_t> words = {r.claimed_sum, r.final_eval};
  for (int i = 0; i < 4; i++) {
    words.push_back((uint32_t)r.digest[i]);
    words.push_back((uint32_t)(r.digest[i] >> 32));
  }
  words.insert(words.end(), rounds_h, rounds_h + 3 * logn);
  return words;
}
std::vector<uint32_t> sumcheck_run(SumcheckBufs& b, const uint32_t* evals, uint32_t logn, cudaStream_t s, uint8_t* pin, double* gpu_s = nullptr) {
  const uint64_t n = 1ull << logn;
  if (!b.ev.p) sumcheck_alloc(b, logn);
  AZK_CU(cudaMemcpyAsync(b.ev.p, evals, 4 * n, cudaMemcpyHostToDevice, s));
  SumcheckOut* h = reinterpret_cast<SumcheckOut*>(pin + align_up(4 * n, 64));
  uint32_t* rounds_h = reinterpret_cast<uint32_t*>(h + 1);
  *h = sumcheck_out_ptrs(b, logn);
  AZK_CU(cudaMemcpyAsync(b.out.p, h, sizeof(SumcheckOut), cudaMemcpyHostToDevice, s));
  std::unique_ptr<GpuTimer> gt;
  if (gpu_s) gt.reset(new GpuTimer(s));
  AZK_CU(launch_sumcheck(b.ev.as<uint32_t>(), logn, b.scratch.as<uint32_t>(), b.out.as<SumcheckOut>(), s));
  if (gt) gt->stop();
  AZK_CU(cudaMemcpyAsync(h, b.out.p, sizeof(SumcheckOut), cudaMemcpyDeviceToHost, s));
  AZK_CU(cudaMemcpyAsync(rounds_h, b.rounds.p, 12ull * logn, cudaMemcpyDeviceToHost, s));
  sync_stream(s);
  if (gt) *gpu_s = gt->seconds();
  return sumcheck_words(*h, rounds_h, logn);
}

// Evict the least recently used cached shape of worker `w` into `dropped` (freed by
// the caller after the server lock is released: a free waits for the whole
// device).  Returns false when the worker caches nothing.
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

// Device memory given back under the lock and freed after it (a free waits for the
// whole device): evicted PCS engines and the buffers of free lane slots.
struct Dropped {
  std::vector<Resident> engines;
  std::vector<SumcheckBufs> tables;
  bool empty() const { return engines.empty() && tables.empty(); }
  void clear() {
    engines.clear();
    tables.clear();
  }
};

// Make room for `bytes` more: this worker's cached shapes first, then idle
// workers' (a worker that runs no job has nothing in flight on its stream), then
// the buffers of free lane slots (reallocated when a table needs them again).
// Called with the lock held; returns whether the bytes fit.
bool make_room(azk_server* sv, int w, uint64_t bytes, Dropped& dropped) {
  while (sv->held + bytes > sv->budget && evict_lru(sv, w, dropped.engines)) {
  }
  for (uint32_t v = 0; v < sv->slots && sv->held + bytes > sv->budget; v++) {
    if ((int)v == w || sv->busy[v]) continue;
    while (sv->held + bytes > sv->budget && evict_lru(sv, (int)v, dropped.engines)) {
    }
  }
  for (size_t k = 0; k < sv->sc_free.size() && sv->held + bytes > sv->budget; k++) {
    SumcheckSlot& sl = *sv->sc_slot[sv->sc_free[k]];
    if (!sl.cap_log) continue;
    sv->held -= sumcheck_table_bytes(sl.cap_log);
    dropped.tables.push_back(std::move(sl.bufs));
    sl.bufs = SumcheckBufs{};
    sl.cap_log = 0;
    sl.grow = false;
  }
  return sv->held + bytes <= sv->budget;
}

// What a worker takes: a group of PCS jobs of one shape, or one sum-check job with
// the lane slot it goes into.
struct Take {
  std::vector<std::shared_ptr<ServeJob>> group;
  int slot = -1;
  bool warm = false;
};

// Called with the server lock held.  Nothing is taken while the front job cannot
// fit; a job larger than the budget never enters the queue.  Evicted memory is
// handed back in `dropped` for the caller to free outside the lock.
bool try_take(azk_server* sv, int w, Take& tk, Dropped& dropped) {
  // this worker's warm-up jobs first; one that cannot fit the budget is dropped
  while (!sv->warm[w].empty()) {
    auto j = sv->warm[w].front();
    auto& cache = sv->cache[w];
    ShapeKey key = shape_of(*j);
    if (!cache.count(key)) {
      const uint32_t cap = shape_capacity(sv, *j);
      const uint64_t bytes = pcs_engine_bytes(j->logn, j->rounds, j->queries, cap) + (sv->domain_logs.count(j->logn) ? 0 : domain_bytes(j->logn));
      if (sv->held + bytes > sv->budget) {
        sv->warm[w].pop_front();
        sv->warm_pending--;
        sv->done_cv.notify_all();
        continue;
      }
      if (sv->domain_logs.insert(j->logn).second) sv->held += domain_bytes(j->logn);
      Resident& r = cache[key];
      r.cap = cap;
      r.bytes = pcs_engine_bytes(j->logn, j->rounds, j->queries, cap);
      sv->held += r.bytes;
    }
    cache[key].last_use = ++sv->tick;
    sv->warm[w].pop_front();
    sv->busy[w] = 1;
    j->state = 1;
    tk.group.assign(std::max<uint32_t>(1, std::min(j->warm_group, cache[key].cap)), j);
    tk.warm = true;
    return true;
  }
  if (sv->queue.empty()) return false;
  // A sum-check costs its worker only a copy into a lane slot, then runs for tens
  // of milliseconds on one warp beside the proofs: while the lane has a free slot,
  // the first queued sum-check goes ahead of the proof jobs, so its digest overlaps
  // them instead of starting after them.  Otherwise the front job; when that is a
  // sum-check and every lane slot holds a table, the first queued proof job (a full
  // lane never holds proof jobs back).
  auto pick = sv->queue.begin();
  if (!sv->sc_free.empty() && sv->queued_sc > 0) {
    while (pick != sv->queue.end() && (*pick)->kind != 1) ++pick;
    if (pick == sv->queue.end()) pick = sv->queue.begin();
  } else if ((*pick)->kind == 1) {
    while (pick != sv->queue.end() && (*pick)->kind == 1) ++pick;
    if (pick == sv->queue.end()) return false;
  }
  // a sum-check goes to a free lane slot; a slot smaller than the table grows
  auto admit_sumcheck = [&](std::deque<std::shared_ptr<ServeJob>>::iterator it) {
    if (sv->sc_free.empty()) return false;
    const std::shared_ptr<ServeJob> sj = *it;
    // the slot leaves the free list first, so making room never takes its buffers
    const int slot = sv->sc_free.back();
    sv->sc_free.pop_back();
    SumcheckSlot& sl = *sv->sc_slot[slot];
    if (sl.cap_log < sj->logn) {
      const uint64_t extra = sumcheck_table_bytes(sj->logn) - (sl.cap_log ? sumcheck_table_bytes(sl.cap_log) : 0);
      if (!make_room(sv, w, extra, dropped)) {
        sv->sc_free.push_back(slot);
        return false;
      }
      sv->held += extra;
      sl.cap_log = sj->logn;  // the worker reallocates before filling the slot
      sl.grow = true;
    }
    sl.job = sj;
    sv->queue.erase(it);
    sv->queued_sc--;
    sv->running++;
    sv->busy[w] = 1;
    sj->state = 1;
    sj->started = std::chrono::steady_clock::now();
    tk.slot = slot;
    return true;
  };
  if ((*pick)->kind == 1) {
    if (admit_sumcheck(pick)) return true;
    // a sum-check taken ahead of the front proof job whose slot cannot grow leaves
    // that proof job to be taken instead
    if (pick == sv->queue.begin()) return false;
    pick = sv->queue.begin();
  }
  std::shared_ptr<ServeJob> j = *pick;
  auto& cache = sv->cache[w];
  const ShapeKey key = shape_of(*j);
  if (!cache.count(key)) {
    const uint32_t cap = shape_capacity(sv, *j);
    const uint64_t eng = pcs_engine_bytes(j->logn, j->rounds, j->queries, cap);
    const uint64_t dom = sv->domain_logs.count(j->logn) ? 0 : domain_bytes(j->logn);
    if (!make_room(sv, w, eng + dom, dropped)) return false;
    if (dom) {
      sv->domain_logs.insert(j->logn);
      sv->held += dom;
    }
    Resident& r = cache[key];
    r.cap = cap;
    r.bytes = eng;
    sv->held += eng;
  }
  Resident& r = cache[key];
  r.last_use = ++sv->tick;
  // the front job and the next queued jobs of its shape, up to the engine's room
  tk.group.clear();
  for (auto it = sv->queue.begin(); it != sv->queue.end() && tk.group.size() < r.cap;) {
    if ((*it)->kind == 0 && shape_of(**it) == key) {
      tk.group.push_back(*it);
      it = sv->queue.erase(it);
    } else {
      ++it;
    }
  }
  const auto now = std::chrono::steady_clock::now();
  for (auto& g : tk.group) {
    g->state = 1;
    g->started = now;
  }
  sv->running += tk.group.size();
  sv->groups++;
  sv->grouped += tk.group.size();
  sv->busy[w] = 1;
  return true;
}

// Publish a finished job (lock held).
void publish(azk_server* sv, ServeJob& j, int outcome, const std::string& error) {
  j.error = error;
  j.state = outcome;
  j.finished = std::chrono::steady_clock::now();
  drop_input(j);
  sv->running--;
  sv->completed++;
  if (j.kind == 0 && outcome == 2) sv->elems += 1ull << j.logn;
  sv->last_finish = j.finished;
}

// Fill a lane slot with a taken sum-check job's table and queue it for a launch.
void lane_submit(azk_server* sv, int slot) {
  SumcheckSlot& sl = *sv->sc_slot[slot];
  ServeJob& j = *sl.job;
  std::string error;
  try {
    AZK_CU(cudaSetDevice(sv->ctx->device));
    if (!sl.bufs.ev.p || sl.grow) sumcheck_alloc(sl.bufs, sl.cap_log);
    sl.grow = false;
    uint8_t* pin = sl.pin.ensure(sumcheck_pinned_bytes(sl.cap_log));
    if (j.zeros)
      std::memset(pin, 0, 4ull << j.logn);
    else
      std::memcpy(pin, job_words(j), 4ull << j.logn);
    drop_input(j);
  } catch (const Error& e) {
    error = e.msg;
  } catch (const std::exception& e) {
    error = e.what();
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  if (!error.empty()) {
    // the slot's memory may be in an unknown state: reallocate it on its next use
    sl.grow = true;
    auto job = sl.job;
    sl.job = nullptr;
    sv->sc_free.push_back(slot);
    if (job->id == 0) {
      job->state = 3;
      sv->running--;
      sv->warm_pending--;
    } else {
      publish(sv, *job, 3, error);
    }
    sv->cv.notify_all();
    sv->done_cv.notify_all();
    return;
  }
  sv->sc_pending.push_back(slot);
  sv->lane_cv.notify_all();
}

// A table of two zeros through a slot on lane stream `s`: a stream's first launch
// and the first device-mapped writes into a slot's staging cost more than later
// ones, so warm-up takes them before serving.
void lane_touch(SumcheckSlot& sl, cudaStream_t s) {
  uint8_t* pin = sl.pin.p;
  SumcheckOut* h = reinterpret_cast<SumcheckOut*>(pin + align_up(4ull << sl.cap_log, 64));
  SumcheckOut* dh = nullptr;
  AZK_CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dh), h, 0));
  uint32_t* drounds = reinterpret_cast<uint32_t*>(dh + 1);
  *h = SumcheckOut{};
  h->r0 = drounds;
  h->r1 = drounds + 1;
  h->challenges = drounds + 2;
  AZK_CU(cudaMemsetAsync(sl.bufs.ev.p, 0, 8, s));
  SumcheckBatch b{};
  b.job[0] = SumcheckJob{sl.bufs.ev.as<uint32_t>(), sl.bufs.scratch.as<uint32_t>(), dh, 1, 0};
  AZK_CU(launch_sumcheck_batch(b, 1, s));
}

// Lane launcher: whenever tables wait and a lane stream is idle, one batched
// launch proves up to kLaneBatch of them.
void lane_launcher(azk_server* sv) {
  cudaSetDevice(sv->ctx->device);
  for (;;) {
    int sid = -1;
    std::vector<int> batch;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->lane_cv.wait(lk, [&] { return (sv->lane_stop && sv->sc_pending.empty()) || (!sv->sc_pending.empty() && !sv->sc_idle.empty()); });
      if (sv->sc_pending.empty()) {
        sv->launcher_done = true;
        sv->lane_cv.notify_all();
        return;
      }
      sid = sv->sc_idle.back();
      sv->sc_idle.pop_back();
      // Tables arriving together (a burst or a backlog: workers stage them one after
      // another) are gathered for up to 1 ms into one launch, so they share launches
      // instead of each taking a lane stream for a whole digest; a table that waits
      // alone goes at once.
      if (sv->sc_pending.size() >= 2 && sv->sc_pending.size() < (size_t)kLaneBatch)
        sv->lane_cv.wait_for(lk, std::chrono::milliseconds(1), [&] { return sv->sc_pending.size() >= (size_t)kLaneBatch || sv->lane_stop; });
      while (!sv->sc_pending.empty() && batch.size() < (size_t)kLaneBatch) {
        batch.push_back(sv->sc_pending.front());
        sv->sc_pending.pop_front();
      }
    }
    SumcheckStream& st = sv->sc_stream[sid];
    st.slots = batch;
    std::string error;
    try {
      SumcheckBatch jobs{};
      for (size_t k = 0; k < batch.size(); k++) {
        SumcheckSlot& sl = *sv->sc_slot[batch[k]];
        const uint32_t logn = sl.job->logn;
        uint8_t* pin = sl.pin.p;
        // results land in the slot's mapped staging, after the table words
        SumcheckOut* h = reinterpret_cast<SumcheckOut*>(pin + align_up(4ull << logn, 64));
        uint32_t* rounds_h = reinterpret_cast<uint32_t*>(h + 1);
        SumcheckOut* dh = nullptr;
        AZK_CU(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dh), h, 0));
        uint32_t* drounds = reinterpret_cast<uint32_t*>(dh + 1);
        *h = SumcheckOut{};
        h->r0 = drounds;
        h->r1 = drounds + logn;
        h->challenges = drounds + 2 * logn;
        std::memset(rounds_h, 0, 12ull * logn);
        AZK_CU(cudaMemcpyAsync(sl.bufs.ev.p, pin, 4ull << logn, cudaMemcpyHostToDevice, st.s));
        jobs.job[k] = SumcheckJob{sl.bufs.ev.as<uint32_t>(), sl.bufs.scratch.as<uint32_t>(), dh, logn, 0};
      }
      AZK_CU(launch_sumcheck_batch(jobs, (uint32_t)batch.size(), st.s));
    } catch (const Error& e) {
      error = e.msg.empty() ? "sum-check launch failed" : e.msg;
    } catch (const std::exception& e) {
      error = e.what();
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!error.empty()) {
      for (int slot : batch) {
        auto job = sv->sc_slot[slot]->job;
        sv->sc_slot[slot]->job = nullptr;
        sv->sc_free.push_back(slot);
        if (job->id == 0) {
          sv->running--;
          sv->warm_pending--;
        } else {
          publish(sv, *job, 3, error);
        }
      }
      sv->sc_idle.push_back(sid);
      sv->cv.notify_all();
      sv->done_cv.notify_all();
      continue;
    }
    sv->sc_inflight.push_back(sid);
    sv->lane_cv.notify_all();
  }
}

// Lane completer: polls the lane streams that run a batch (cudaStreamQuery every
// 200 us, nothing queued behind the kernels), and publishes a finished batch's
// results from its slots' mapped staging.
void lane_completer(azk_server* sv) {
  cudaSetDevice(sv->ctx->device);
  for (;;) {
    std::vector<int> inflight;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->lane_cv.wait(lk, [&] { return !sv->sc_inflight.empty() || sv->launcher_done; });
      if (sv->sc_inflight.empty()) return;
      inflight.assign(sv->sc_inflight.begin(), sv->sc_inflight.end());
    }
    std::vector<std::pair<int, std::string>> finished;  // (stream, error)
    for (int sid : inflight) {
      const cudaError_t e = cudaStreamQuery(sv->sc_stream[sid].s);
      if (e == cudaErrorNotReady) continue;
      if (e != cudaSuccess) cudaGetLastError();
      finished.emplace_back(sid, e == cudaSuccess ? std::string() : std::string("sum-check batch failed: ") + cudaGetErrorString(e));
    }
    if (finished.empty()) {
      std::this_thread::sleep_for(std::chrono::microseconds(200));
      continue;
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    for (auto& [sid, error] : finished) {
      SumcheckStream& st = sv->sc_stream[sid];
      for (const int slot : st.slots) {
        SumcheckSlot& sl = *sv->sc_slot[slot];
        auto job = sl.job;
        sl.job = nullptr;
        sv->sc_free.push_back(slot);
        if (job->id == 0) {  // a warm-up table
          job->state = error.empty() ? 2 : 3;
          sv->running--;
          sv->warm_pending--;
          continue;
        }
        if (error.empty()) {
          const SumcheckOut* h = reinterpret_cast<const SumcheckOut*>(sl.pin.p + align_up(4ull << job->logn, 64));
          const std::vector<uint32_t> words = sumcheck_words(*h, reinterpret_cast<const uint32_t*>(h + 1), job->logn);
          job->result.resize(4 * words.size());
          std::memcpy(job->result.data(), words.data(), job->result.size());
        }
        publish(sv, *job, error.empty() ? 2 : 3, error);
      }
      st.slots.clear();
      sv->sc_inflight.erase(std::find(sv->sc_inflight.begin(), sv->sc_inflight.end(), sid));
      sv->sc_idle.push_back(sid);
    }
    sv->cv.notify_all();
    sv->done_cv.notify_all();
    sv->lane_cv.notify_all();
  }
}

void worker_loop(azk_server* sv, int w) {
  cudaSetDevice(sv->ctx->device);
  // everything this worker runs (uploads and proof kernels) goes on its one stream:
  // its groups run one at a time, and one stream per worker keeps each worker on
  // its own hardware work queue (see azk_server_create)
  cudaStream_t s = sv->streams[w];
  Staging staging;
  for (;;) {
    Take tk;
    Resident* res = nullptr;
    Dropped dropped;  // evicted memory, freed below without the lock
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      bool got = false;
      for (;;) {
        if (sv->stop && sv->queue.empty() && sv->warm[w].empty()) break;
        got = try_take(sv, w, tk, dropped);
        if (got) break;
        if (!dropped.empty()) {  // free what was evicted, then look again
          lk.unlock();
          dropped.clear();
          lk.lock();
          continue;
        }
        sv->cv.wait(lk);
      }
      if (!got) break;
      if (tk.slot < 0) res = &sv->cache[w][shape_of(*tk.group[0])];
    }
    dropped.clear();
    if (tk.slot >= 0) {  // a sum-check: into the lane, and on to the next job
      lane_submit(sv, tk.slot);
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->busy[w] = 0;
      sv->cv.notify_all();
      continue;
    }
    // the outcome is published under the lock together with the finish time, so a
    // poll never sees a finished job without its latency
    int outcome = 2;
    std::string error;
    try {
      run_pcs_group(sv, *res, tk.group, staging, s);
    } catch (const Error& e) {
      error = e.msg;
      outcome = 3;
    } catch (const std::exception& e) {
      error = e.what();
      outcome = 3;
    }
    std::vector<Resident> failed;  // a failed group's shape, freed without the lock
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->busy[w] = 0;
      if (outcome == 3) {  // drop the shape's memory: it may be in an unknown state
        auto it = sv->cache[w].find(shape_of(*tk.group[0]));
        if (it != sv->cache[w].end()) {
          sv->held -= it->second.bytes;
          failed.push_back(std::move(it->second));
          sv->cache[w].erase(it);
        }
      }
      if (tk.warm) {  // warm-up jobs are not results anyone polls
        tk.group[0]->state = outcome;
        sv->warm_pending--;
      } else {
        for (auto& j : tk.group) publish(sv, *j, outcome, error);
      }
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

uint64_t submit(azk_server* sv, std::shared_ptr<ServeJob> j, uint64_t bytes) {
  std::lock_guard<std::mutex> lk(sv->mu);
  require(bytes <= sv->budget, AZK_ERR_HBM_BUDGET,
          "job needs " + std::to_string(bytes) + " device bytes, more than the server's HBM budget of " + std::to_string(sv->budget));
  j->id = sv->next_id++;
  j->submitted = std::chrono::steady_clock::now();
  if (!sv->any_submit) {
    sv->first_submit = j->submitted;
    sv->any_submit = true;
  }
  sv->jobs[j->id] = j;
  sv->queue.push_back(j);
  if (j->kind == 1) sv->queued_sc++;
  sv->cv.notify_all();
  return j->id;
}

// The submission entry points: arguments checked (a non-canonical word is refused
// here, before the job is queued), then the words copied into the job or, with
// `borrow`, only their address kept: the worker that takes the job reads them into
// its page-locked staging.
uint64_t submit_pcs(azk_server* sv, uint32_t logn, uint32_t log_blowup, uint32_t queries, uint32_t rounds, const uint32_t* coeffs,
                    uint64_t count, const uint8_t pub[32], const uint64_t* job_id, bool borrow) {
  layout(sv && coeffs && pub && job_id);
  validate_params(logn, log_blowup, queries, 0, rounds);
  layout(count >= 1 && count <= (1ull << logn));
  layout(all_canonical(coeffs, 4 * count), "input contains a non-canonical field element");
  auto j = std::make_shared<ServeJob>();
  j->kind = 0;
  j->logn = logn;
  j->rounds = rounds;
  j->queries = queries;
  j->log_blowup = log_blowup;
  if (borrow)
    j->borrowed = coeffs;
  else
    j->input.assign(coeffs, coeffs + 4 * count);
  j->count = count;
  std::memcpy(j->pub, pub, 32);
  return submit(sv, j, pcs_engine_bytes(logn, rounds, queries, 1) + domain_bytes(logn));
}

uint64_t submit_sumcheck(azk_server* sv, const uint32_t* evals, uint64_t count, const uint64_t* job_id, bool borrow) {
  layout(sv && evals && job_id);
  // M31MultilinearSumcheckProofBuilderV1.prove preconditions (SumcheckOracle.swift:803-807)
  layout(count > 1 && is_pow2(count) && count <= (1ull << 28));
  layout(all_canonical(evals, count), "input contains a non-canonical field element");
  auto j = std::make_shared<ServeJob>();
  j->kind = 1;
  j->logn = ilog2(count);
  if (borrow)
    j->borrowed = evals;
  else
    j->input.assign(evals, evals + count);
  return submit(sv, j, sumcheck_table_bytes(j->logn));
}

}  // namespace

extern "C" {

azk_status azk_sumcheck_prove(azk_ctx* ctx, const uint32_t* evals, uint64_t count, uint32_t* sums0, uint32_t* sums1, uint32_t* challenges,
                              uint32_t* claimed_sum, uint32_t* final_eval, uint8_t digest[32], azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && evals && sums0 && sums1 && challenges && claimed_sum && final_eval && digest);
    // preconditions of M31MultilinearSumcheckProofBuilderV1.prove (SumcheckOracle.swift:803-807)
    layout(count > 1 && is_pow2(count) && count <= (1ull << 28), "evaluation count must be a power of two greater than one");
    layout(all_canonical(evals, count), "input contains a non-canonical field element");
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
    // a group proves few instances: the single-tree table (measured on the serving
    // mix: the lowest latency per job at a throughput equal to the batch table's
    // within run-to-run spread)
    sv->sched = resolve_schedule(schedule, kTuned_pcs_single, kTunedThreads_pcs_single);
    sv->budget = hbm_budget_bytes;
    sv->slots = slots;
    sv->cache.resize(slots);
    sv->busy.assign(slots, 0);
    sv->warm.resize(slots);
    AZK_CU(cudaSetDevice(ctx->device));
    // The workers' streams are created first, one after another, so that with up to
    // CUDA_DEVICE_MAX_CONNECTIONS (32) workers each lands on its own hardware work
    // queue.  Streams that share a queue wait on each other's dependent launches;
    // nothing here issues a launch that waits long on an earlier one in its stream
    // (the sum-check lane proves a table in one launch).  Priorities: the lane's
    // tables (one CTA each, the longest jobs) take the first free SM slot, then the
    // workers' launches (a job's input scan ahead of default-priority work).
    int prio_lo = 0, prio_hi = 0;
    AZK_CU(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    const int prio_worker = prio_hi < prio_lo ? prio_hi + 1 : prio_hi;
    sv->streams.assign(slots, nullptr);
    for (uint32_t w = 0; w < slots; w++) AZK_CU(cudaStreamCreateWithPriority(&sv->streams[w], cudaStreamNonBlocking, prio_worker));
    sv->sc_stream.resize(kLaneStreams);
    for (int k = 0; k < kLaneStreams; k++) {
      AZK_CU(cudaStreamCreateWithPriority(&sv->sc_stream[k].s, cudaStreamNonBlocking, prio_hi));
      sv->sc_idle.push_back(k);
    }
    for (int k = 0; k < kLaneSlots; k++) {
      sv->sc_slot.push_back(std::make_unique<SumcheckSlot>());
      sv->sc_free.push_back(kLaneSlots - 1 - k);
    }
    for (uint32_t w = 0; w < slots; w++) sv->workers.emplace_back(worker_loop, sv.get(), (int)w);
    sv->sc_launcher = std::thread(lane_launcher, sv.get());
    sv->sc_completer = std::thread(lane_completer, sv.get());
    *out = sv.release();
  });
}

azk_status azk_server_submit_pcs(azk_server* sv, uint32_t logn, uint32_t log_blowup, uint32_t queries, uint32_t rounds, const uint32_t* coeffs,
                                 uint64_t count, const uint8_t pub[32], uint64_t* job_id) {
  return guarded(sv ? sv->ctx : nullptr, [&] { *job_id = submit_pcs(sv, logn, log_blowup, queries, rounds, coeffs, count, pub, job_id, false); });
}

azk_status azk_server_submit_pcs_nocopy(azk_server* sv, uint32_t logn, uint32_t log_blowup, uint32_t queries, uint32_t rounds,
                                        const uint32_t* coeffs, uint64_t count, const uint8_t pub[32], uint64_t* job_id) {
  return guarded(sv ? sv->ctx : nullptr, [&] { *job_id = submit_pcs(sv, logn, log_blowup, queries, rounds, coeffs, count, pub, job_id, true); });
}

azk_status azk_server_warm(azk_server* sv, const uint32_t* pcs_logn, const uint32_t* pcs_rounds, uint32_t n_pcs, uint32_t log_blowup,
                           uint32_t queries, const uint32_t* sumcheck_logn, uint32_t n_sumcheck) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv && (n_pcs == 0 || (pcs_logn && pcs_rounds)) && (n_sumcheck == 0 || sumcheck_logn));
    for (uint32_t i = 0; i < n_pcs; i++) validate_params(pcs_logn[i], log_blowup, queries, 0, pcs_rounds[i]);
    uint32_t sc_log = 0;
    std::vector<uint32_t> sc_logs;  // listed tables that fit the budget
    for (uint32_t i = 0; i < n_sumcheck; i++) {
      layout(sumcheck_logn[i] >= 1 && sumcheck_logn[i] <= 28);
      if (sumcheck_table_bytes(sumcheck_logn[i]) > sv->budget) continue;
      sc_logs.push_back(sumcheck_logn[i]);
      sc_log = std::max(sc_log, sumcheck_logn[i]);
    }
    // the lane's table slots for the largest listed table, as many as fit the budget
    if (sc_log) {
      AZK_CU(cudaSetDevice(sv->ctx->device));
      for (int k = 0; k < kLaneSlots; k++) {
        SumcheckSlot* sl = nullptr;
        {
          // a free slot is taken out of the free list while it is allocated
          std::lock_guard<std::mutex> lk(sv->mu);
          auto it = std::find(sv->sc_free.begin(), sv->sc_free.end(), k);
          if (it == sv->sc_free.end()) continue;
          sl = sv->sc_slot[k].get();
          if (sl->cap_log >= sc_log && !sl->grow) continue;
          const uint64_t extra = sumcheck_table_bytes(sc_log) - (sl->cap_log ? sumcheck_table_bytes(sl->cap_log) : 0);
          if (sv->held + extra > sv->budget) break;
          sv->held += extra;
          sl->cap_log = sc_log;
          sv->sc_free.erase(it);
        }
        try {
          sumcheck_alloc(sl->bufs, sc_log);
          sl->grow = false;
          sl->pin.ensure(sumcheck_pinned_bytes(sc_log));
          lane_touch(*sl, sv->sc_stream[k % kLaneStreams].s);
          sync_stream(sv->sc_stream[k % kLaneStreams].s);  // the slot's staging is idle again
        } catch (...) {
          std::lock_guard<std::mutex> lk(sv->mu);
          sl->grow = true;
          sv->sc_free.push_back(k);
          throw;
        }
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->sc_free.push_back(k);
      }
    }
    std::unique_lock<std::mutex> lk(sv->mu);
    for (uint32_t w = 0; w < sv->slots; w++) {
      for (uint32_t i = 0; i < n_pcs; i++) {
        ServeJob shape;
        shape.logn = pcs_logn[i];
        shape.rounds = pcs_rounds[i];
        shape.queries = queries;
        shape.log_blowup = log_blowup;
        // one group of each size the shape can take: a group size's first run
        // builds the engine's FFT work lists for it (device allocations) and
        // captures its graph, and either, in the middle of serving, waits for the
        // whole device, long sum-check kernels included
        const uint32_t cap = shape_capacity(sv, shape);
        for (uint32_t m = cap; m >= 1; m--) {
          auto j = std::make_shared<ServeJob>();  // id 0: a warm-up job
          j->kind = 0;
          j->logn = shape.logn;
          j->rounds = shape.rounds;
          j->queries = queries;
          j->log_blowup = log_blowup;
          j->warm_group = m;
          // all 2^logn coefficients (zeros): the worker's pinned staging grows to a
          // full group of the shape's largest inputs now, not in the middle of
          // serving, where freeing the smaller buffer would wait for the whole device
          j->zeros = true;
          j->count = 1ull << j->logn;
          sv->warm[w].push_back(j);
          sv->warm_pending++;
        }
      }
    }
    // one table of zeros per listed size through the lane (kernels loaded before serving)
    for (uint32_t lg : sc_logs) {
      auto j = std::make_shared<ServeJob>();
      j->kind = 1;
      j->logn = lg;
      j->zeros = true;
      sv->queue.push_front(j);
      sv->queued_sc++;
      sv->warm_pending++;
    }
    sv->cv.notify_all();
    sv->done_cv.wait(lk, [&] { return sv->warm_pending == 0; });
  });
}

azk_status azk_server_submit_sumcheck(azk_server* sv, const uint32_t* evals, uint64_t count, uint64_t* job_id) {
  return guarded(sv ? sv->ctx : nullptr, [&] { *job_id = submit_sumcheck(sv, evals, count, job_id, false); });
}

azk_status azk_server_submit_sumcheck_nocopy(azk_server* sv, const uint32_t* evals, uint64_t count, uint64_t* job_id) {
  return guarded(sv ? sv->ctx : nullptr, [&] { *job_id = submit_sumcheck(sv, evals, count, job_id, true); });
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

azk_status azk_server_group_stats(azk_server* sv, uint64_t* groups, uint64_t* grouped_jobs) {
  return guarded(sv ? sv->ctx : nullptr, [&] {
    layout(sv != nullptr);
    std::lock_guard<std::mutex> lk(sv->mu);
    if (groups) *groups = sv->groups;
    if (grouped_jobs) *grouped_jobs = sv->grouped;
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
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->lane_stop = true;
  }
  sv->lane_cv.notify_all();
  if (sv->sc_launcher.joinable()) sv->sc_launcher.join();
  if (sv->sc_completer.joinable()) sv->sc_completer.join();
  for (auto& st : sv->sc_stream)
    if (st.s) cudaStreamDestroy(st.s);
  for (auto st : sv->streams)
    if (st) cudaStreamDestroy(st);
  delete sv;
}

}  // extern "C"
