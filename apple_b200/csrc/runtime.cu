// Context, buffers, domain tables and the primitive plans of the C ABI:
// Keccak-f batch, SHA3/Keccak batch hashing, raw/prehashed Merkle commitment,
// Circle FFT codeword, single folds and fold chains.
#include <algorithm>
#include <cstdlib>

#include "azk_field.cuh"
#include "azk_runtime.h"
#include "azk_tuned.h"

using namespace azk;

static thread_local std::string g_thread_error;

void azk::set_error(const azk_ctx* ctx, const std::string& msg) {
  g_thread_error = msg;
  if (ctx) {
    auto* c = const_cast<azk_ctx*>(ctx);
    std::lock_guard<std::mutex> lk(c->mu);
    c->last_error = msg;
  }
}

const azk_ctx::Domain& azk::domain_tables(azk_ctx* ctx, uint32_t logn) {
  require(logn >= 1 && logn <= 26, AZK_ERR_INVALID_INPUT_LAYOUT, "circle domain log size must be in 1...26");
  std::lock_guard<std::mutex> lk(ctx->mu);
  auto it = ctx->domains.find(logn);
  if (it != ctx->domains.end()) return it->second;
  uint64_t n = 1ull << logn;
  azk_ctx::Domain d;
  AZK_CU(cudaMalloc(&d.tw, 4 * 2 * n));  // twiddles, then their doubled copy at tw + N
  AZK_CU(cudaMalloc(&d.inv, 4 * (n - 1 + 1)));
  AZK_CU(launch_domain_tables(logn, d.tw, d.inv, ctx->stream));
  sync_stream(ctx->stream);
  return ctx->domains.emplace(logn, d).first->second;
}

Sched azk::resolve_schedule(const azk_schedule* s, const uint8_t* defaults, const uint16_t* default_threads) {
  Sched r;
  bool any_layer = false, any_threads = false;
  if (s) {
    if (s->treelet_log) r.tile_log = s->treelet_log;
    if (s->group_log) r.group_log = s->group_log;
    if (s->threads) r.threads = s->threads;
    r.graph = s->use_graph != 0;
    r.persistent_trees = s->persistent_trees != 0;
    for (int i = 0; i < 32; i++) {
      r.layer_tile[i] = s->layer_treelet[i];
      any_layer |= r.layer_tile[i] != 0;
      require(r.layer_tile[i] <= 13, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "layer treelet depth must be in 0...13");
      const uint16_t th = s->layer_threads[i];
      require(th == 0 || th == 128 || th == 256 || th == 512, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "layer threads must be 0, 128, 256 or 512");
      r.layer_threads[i] = th;
      any_threads |= th != 0;
    }
  }
  if (defaults && !any_layer && !(s && s->treelet_log))
    for (int i = 0; i < 32; i++) r.layer_tile[i] = defaults[i] <= 13 ? defaults[i] : 13;
  if (default_threads && !any_threads && !(s && s->threads))
    for (int i = 0; i < 32; i++) r.layer_threads[i] = (default_threads[i] == 128 || default_threads[i] == 256 || default_threads[i] == 512) ? default_threads[i] : 0;
  require(r.tile_log >= 1 && r.tile_log <= 13, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "treelet_log must be in 1...13");
  if (r.group_log > r.tile_log) r.group_log = r.tile_log;
  require(r.group_log >= 1, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "group_log must be >= 1");
  require(r.threads == 128 || r.threads == 256 || r.threads == 512, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "threads must be 128, 256 or 512");
  return r;
}

// ---------------------------------------------------------------------------
// FFT plans
// ---------------------------------------------------------------------------
namespace {
// cuMemGetAddressRange through the runtime's driver entry point (no link against
// the driver library): CUresult (*)(CUdeviceptr* base, size_t* size, CUdeviceptr p).
using MemRangeFn = int (*)(unsigned long long*, size_t*, unsigned long long);
MemRangeFn mem_range_fn() {
  static MemRangeFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<MemRangeFn>(f);
  }();
  return fn;
}
}  // namespace

void azk::require_device_range(const void* p, uint64_t off, uint64_t bytes) {
  layout(p != nullptr, "null device pointer");
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  layout(a + off >= a && a + off + bytes >= a + off, "device range overflows");
  MemRangeFn fn = mem_range_fn();
  require(fn != nullptr, AZK_ERR_COMMAND_EXECUTION_FAILED, "cuMemGetAddressRange is not available from the driver");
  unsigned long long base = 0;
  size_t size = 0;
  if (fn(&base, &size, (unsigned long long)(a + off)) != 0)
    fail(AZK_ERR_INVALID_INPUT_LAYOUT, "resident buffer is not device memory of this context");
  layout(a + off + bytes <= base + size, "resident buffer range runs past the end of its device allocation");
}

void FftPlan::build(const std::vector<FftJob>& transforms, const std::vector<uint8_t>& narrow_flags) {
  jobs.clear();
  work.clear();
  narrow.assign(transforms.size(), 0);
  for (size_t i = 0; i < transforms.size() && i < narrow_flags.size(); i++) narrow[i] = narrow_flags[i] ? 1 : 0;
  uint32_t max_passes = 0;
  for (auto& t : transforms) max_passes = std::max(max_passes, fft_high_chunks(t.logn) + 1);
  std::array<uint64_t, kFftKinds> zero{};
  part_off.assign(max_passes, zero);
  part_cnt.assign(max_passes, zero);
  inst_range.assign(max_passes, std::vector<std::pair<uint64_t, uint64_t>>(transforms.size(), {0, 0}));
  inst_kind.assign(max_passes, std::vector<uint8_t>(transforms.size(), 0));
  std::vector<std::vector<uint32_t>> job_at(max_passes, std::vector<uint32_t>(transforms.size(), UINT32_MAX));
  for (size_t i = 0; i < transforms.size(); i++) {
    uint32_t passes = fft_high_chunks(transforms[i].logn) + 1;
    for (uint32_t p = 0; p < passes; p++) {
      FftJob j = transforms[i];
      j.pass = p;
      job_at[max_passes - passes + p][i] = (uint32_t)jobs.size();
      jobs.push_back(j);
    }
  }
  for (uint32_t step = 0; step < max_passes; step++) {
    for (uint32_t kind = 0; kind < kFftKinds; kind++) {
      part_off[step][kind] = work.size();
      for (size_t i = 0; i < transforms.size(); i++) {
        uint32_t jid = job_at[step][i];
        if (jid == UINT32_MAX) continue;
        const FftJob& j = jobs[jid];
        if (fft_pass_kind(j.logn, j.pass, narrow[i] != 0) != kind) continue;
        uint64_t tiles = fft_kind_tiles(j.logn, j.pass, kind);
        inst_range[step][i] = {work.size(), tiles};
        inst_kind[step][i] = (uint8_t)kind;
        for (uint64_t t = 0; t < tiles; t++) work.push_back(make_uint2(jid, (uint32_t)t));
      }
      part_cnt[step][kind] = work.size() - part_off[step][kind];
    }
  }
}
// Device lists keep their allocation when the new ones fit (a server group of
// another size rebuilds the lists without an allocation, which would wait for the
// whole device).
void FftPlan::upload(cudaStream_t s) {
  const uint64_t jb = std::max<size_t>(1, jobs.size()) * sizeof(FftJob), wb = std::max<size_t>(1, work.size()) * sizeof(uint2);
  if (d_jobs.bytes < jb) d_jobs.alloc(jb, "fft jobs");
  if (d_work.bytes < wb) d_work.alloc(wb, "fft work");
  if (!d_status.p) {
    d_status.alloc(16, "fft status");
    AZK_CU(cudaMemsetAsync(d_status.p, 0, 16, s));
  }
  if (!jobs.empty()) AZK_CU(cudaMemcpyAsync(d_jobs.p, jobs.data(), jobs.size() * sizeof(FftJob), cudaMemcpyHostToDevice, s));
  if (!work.empty()) AZK_CU(cudaMemcpyAsync(d_work.p, work.data(), work.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
}
void FftPlan::launch_step(size_t step, cudaStream_t s) const {
  for (uint32_t kind = 0; kind < kFftKinds; kind++)
    AZK_CU(launch_fft_pass(d_jobs.as<FftJob>(), d_work.as<uint2>() + part_off[step][kind], (uint32_t)part_cnt[step][kind], kind,
                           d_status.as<uint32_t>(), s));
}
void FftPlan::launch_step_for(size_t step, size_t t, cudaStream_t s) const {
  auto r = inst_range[step][t];
  AZK_CU(launch_fft_pass(d_jobs.as<FftJob>(), d_work.as<uint2>() + r.first, (uint32_t)r.second, inst_kind[step][t], d_status.as<uint32_t>(), s));
}
void FftPlan::check_status(cudaStream_t s, uint32_t* host_word) {
  if (!d_status.p) return;
  uint32_t local = 0;
  uint32_t* f = host_word ? host_word : &local;
  AZK_CU(cudaMemcpyAsync(f, d_status.p, 4, cudaMemcpyDeviceToHost, s));
  sync_stream(s);
  if (*f) {
    AZK_CU(cudaMemsetAsync(d_status.p, 0, 4, s));
    fail(AZK_ERR_DEVICE_TIMEOUT, "a Circle FFT pass gave up waiting for its bulk tile copies");
  }
}

// ---------------------------------------------------------------------------
// Monomial -> FFT basis (host preprocessing of CircleCodewordPlan.execute(polynomial:))
// ---------------------------------------------------------------------------
namespace {
struct Q {
  uint32_t a, b, c, d;
};
inline Q qadd(Q x, Q y) { return {m31_add(x.a, y.a), m31_add(x.b, y.b), m31_add(x.c, y.c), m31_add(x.d, y.d)}; }
inline Q qsub(Q x, Q y) { return {m31_sub(x.a, y.a), m31_sub(x.b, y.b), m31_sub(x.c, y.c), m31_sub(x.d, y.d)}; }
inline Q qscale(Q x, uint32_t s) { return {m31_mul(x.a, s), m31_mul(x.b, s), m31_mul(x.c, s), m31_mul(x.d, s)}; }
inline bool qzero(Q x) { return !(x.a | x.b | x.c | x.d); }

// Chebyshev coefficients -> line FFT basis, recursively on halves.
std::vector<Q> chebyshev_to_line(const std::vector<Q>& c) {
  if (c.size() == 1) return c;
  size_t half = c.size() / 2;
  std::vector<Q> lo(c.begin(), c.begin() + half), hi(half, Q{0, 0, 0, 0});
  hi[0] = c[half];
  for (size_t i = 1; i < half; i++) hi[i] = qscale(c[half + i], 2);
  for (size_t li = 1; li < half; li++) lo[li] = qsub(lo[li], qscale(hi[half - li], kInv2));
  auto a = chebyshev_to_line(lo), b = chebyshev_to_line(hi);
  a.insert(a.end(), b.begin(), b.end());
  return a;
}
// Monomials -> Chebyshev (x^d expanded by repeated multiplication by x) -> line basis.
std::vector<Q> line_basis(const uint32_t* m, uint64_t count, uint64_t capacity) {
  std::vector<Q> ch(capacity, Q{0, 0, 0, 0});
  if (count == 0) return ch;
  std::vector<uint32_t> power = {1};
  for (uint64_t deg = 0; deg < count; deg++) {
    Q cf = {m[4 * deg], m[4 * deg + 1], m[4 * deg + 2], m[4 * deg + 3]};
    if (!qzero(cf))
      for (size_t i = 0; i < power.size(); i++)
        if (power[i]) ch[i] = qadd(ch[i], qscale(cf, power[i]));
    if (deg + 1 < count) {
      std::vector<uint32_t> nx(power.size() + 1, 0);
      for (size_t i = 0; i < power.size(); i++) {
        uint32_t v = power[i];
        if (!v) continue;
        if (i == 0) {
          nx[1] = m31_add(nx[1], v);
        } else {
          uint32_t h = m31_mul(v, kInv2);
          nx[i - 1] = m31_add(nx[i - 1], h);
          nx[i + 1] = m31_add(nx[i + 1], h);
        }
      }
      power.swap(nx);
    }
  }
  return chebyshev_to_line(ch);
}
}  // namespace

std::vector<uint32_t> azk::fft_basis_from_monomials(uint32_t logn, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny) {
  uint64_t half = 1ull << (logn - 1);
  layout(nx <= half && ny <= half && (nx || ny));
  layout(all_canonical(x, 4 * nx));
  layout(all_canonical(y, 4 * ny));
  auto xl = line_basis(x, nx, half), yl = line_basis(y, ny, half);
  std::vector<uint32_t> out(8 * half);
  for (uint64_t i = 0; i < half; i++) {
    std::memcpy(&out[8 * i], &xl[i], 16);
    std::memcpy(&out[8 * i + 4], &yl[i], 16);
  }
  return out;
}

// ---------------------------------------------------------------------------
// Context and buffers
// ---------------------------------------------------------------------------
extern "C" {

azk_status azk_ctx_create(int device, azk_ctx** out) {
  return guarded(nullptr, [&] {
    layout(out != nullptr);
    // Streams beyond the device's hardware work queues share queues, and a long
    // kernel then blocks unrelated streams behind it (the server runs one stream
    // per worker).  The queue count is read when CUDA initialises, so this only
    // takes effect when this library is the first CUDA user of the process, and
    // never overrides a value the caller set.
    setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
      cudaGetLastError();
      fail(AZK_ERR_UNAVAILABLE, "no CUDA device is available");
    }
    require(device >= 0 && device < n, AZK_ERR_UNAVAILABLE, "CUDA device index out of range");
    cudaDeviceProp prop;
    AZK_CU(cudaGetDeviceProperties(&prop, device));
    require(prop.major == 10, AZK_ERR_UNAVAILABLE, "this library is built for sm_100a (B200); found compute capability " +
                                                       std::to_string(prop.major) + "." + std::to_string(prop.minor));
    AZK_CU(cudaSetDevice(device));
    AZK_CU(prepare_tree_kernels());
    AZK_CU(prepare_fft_kernels());
    auto* c = new azk_ctx();
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    c->cc_major = prop.major;
    c->cc_minor = prop.minor;
    c->total_mem = prop.totalGlobalMem;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      fail(AZK_ERR_COMMAND_EXECUTION_FAILED, "failed to create a CUDA stream");
    }
    *out = c;
  });
}

void azk_ctx_destroy(azk_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  for (auto& kv : ctx->domains) {
    cudaFree(kv.second.tw);
    cudaFree(kv.second.inv);
  }
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* azk_last_error_message(const azk_ctx* ctx) {
  if (ctx) return ctx->last_error.c_str();
  return g_thread_error.c_str();
}

azk_status azk_ctx_device_info(azk_ctx* ctx, int* sm_count, uint64_t* total_bytes, int* cc_major, int* cc_minor) {
  return guarded(ctx, [&] {
    layout(ctx != nullptr);
    if (sm_count) *sm_count = ctx->sm_count;
    if (total_bytes) *total_bytes = ctx->total_mem;
    if (cc_major) *cc_major = ctx->cc_major;
    if (cc_minor) *cc_minor = ctx->cc_minor;
  });
}

azk_status azk_buf_alloc(azk_ctx* ctx, uint64_t bytes, void** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    AZK_CU(cudaSetDevice(ctx->device));
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      cudaGetLastError();
      fail(AZK_ERR_FAILED_TO_CREATE_BUFFER, "Failed to create device buffer of length " + std::to_string(bytes));
    }
    *out = p;
  });
}
azk_status azk_buf_free(azk_ctx* ctx, void* ptr) {
  return guarded(ctx, [&] {
    if (ptr) AZK_CU(cudaFree(ptr));
  });
}
azk_status azk_buf_upload(azk_ctx* ctx, void* dst, uint64_t off, const void* src, uint64_t bytes) {
  return guarded(ctx, [&] {
    layout(ctx && dst && (src || !bytes));
    if (bytes) AZK_CU(cudaMemcpy(static_cast<uint8_t*>(dst) + off, src, bytes, cudaMemcpyHostToDevice));
  });
}
azk_status azk_buf_download(azk_ctx* ctx, void* dst, const void* src, uint64_t off, uint64_t bytes) {
  return guarded(ctx, [&] {
    layout(ctx && src && (dst || !bytes));
    if (bytes) AZK_CU(cudaMemcpy(dst, static_cast<const uint8_t*>(src) + off, bytes, cudaMemcpyDeviceToHost));
  });
}
azk_status azk_buf_zero(azk_ctx* ctx, void* dst, uint64_t bytes) {
  return guarded(ctx, [&] {
    layout(ctx && dst);
    if (bytes) AZK_CU(cudaMemset(dst, 0, bytes));
  });
}
azk_status azk_synchronize(azk_ctx* ctx) {
  return guarded(ctx, [&] {
    layout(ctx != nullptr);
    AZK_CU(cudaDeviceSynchronize());
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Plans
// ---------------------------------------------------------------------------
struct azk_keccakf_plan {
  azk_ctx* ctx;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint64_t count, in_stride, out_stride;
  uint32_t threads;
  DevBuf in, out;
  ~azk_keccakf_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

struct azk_hash_plan {
  azk_ctx* ctx;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint64_t count, stride, length, out_stride;
  uint32_t suffix, threads;
  DevBuf in, out;
  ~azk_hash_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

struct azk_merkle_plan {
  azk_ctx* ctx;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint64_t count, stride, length;
  uint32_t logn, tile_log, threads = 256;
  DevBuf leaves, leaf_digests, inner, counters, job, work, root, idx, paths;
  TreeJob h_job{};
  std::vector<uint2> h_work;
  bool committed = false;
  ~azk_merkle_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

struct azk_merkle_prehashed_plan {
  azk_ctx* ctx;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint64_t count;
  uint32_t logn, tile_log;
  DevBuf staging, inner, counters, job, work, root;
  TreeJob h_job{};
  ~azk_merkle_prehashed_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

struct azk_codeword_plan {
  azk_ctx* ctx;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint32_t logn;
  DevBuf coeff, out;
  FftPlan fft;
  azk_witness_plan* wit = nullptr;  // monomials -> FFT basis on the device (made on first use)
  ~azk_codeword_plan() {
    if (wit) azk_witness_plan_destroy(wit);
    if (s) cudaStreamDestroy(s);
  }
};
// Host monomial columns -> interleaved FFT-basis coefficients in device memory
// `dout` (2 * capacity QM31), through the witness plan's kernels; returns when done.
static void witness_columns_to_device(azk_witness_plan* w, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny, void* dout);

static cudaStream_t new_stream() {
  cudaStream_t s;
  AZK_CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

extern "C" {

// ---- Keccak-f ----
azk_status azk_keccakf_plan_create(azk_ctx* ctx, uint64_t count, uint64_t in_stride, uint64_t out_stride, uint32_t threads, azk_keccakf_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // KeccakF1600PermutationBatchPlan.validate (KeccakF1600PermutationBatcher.swift:213-222)
    layout(count > 0 && in_stride >= 200 && out_stride >= 200 && in_stride % 8 == 0 && out_stride % 8 == 0 && count <= 0xFFFFFFFFull);
    require(threads == 0 || threads == 64 || threads == 128 || threads == 256, AZK_ERR_INVALID_KERNEL_CONFIGURATION,
            "threads per block must be 64, 128 or 256");
    AZK_CU(cudaSetDevice(ctx->device));
    auto p = std::make_unique<azk_keccakf_plan>();
    p->ctx = ctx;
    p->count = count;
    p->in_stride = in_stride;
    p->out_stride = out_stride;
    p->threads = threads;
    p->in.alloc(count * in_stride, "KeccakF1600Permutation.Input");
    p->out.alloc(count * out_stride, "KeccakF1600Permutation.Output");
    p->s = new_stream();
    *out = p.release();
  });
}

static void keccakf_run(azk_keccakf_plan* p, const uint8_t* din, uint8_t* dout, azk_stats* st, const Timer& t) {
  GpuTimer g(p->s);
  AZK_CU(launch_keccak_permute(din, p->in_stride, dout, p->out_stride, p->count, p->threads, p->s));
  uint64_t sub = t.ns();
  g.stop();
  double gs = g.seconds();
  fill_stats(st, t, sub, gs);
}

azk_status azk_keccakf_plan_permute(azk_keccakf_plan* p, const void* host_states, void* host_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && host_states && host_out);
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->in.p, host_states, p->count * p->in_stride, cudaMemcpyHostToDevice, p->s));
    keccakf_run(p, p->in.as<uint8_t>(), p->out.as<uint8_t>(), nullptr, t);
    AZK_CU(cudaMemcpyAsync(host_out, p->out.p, p->count * p->out_stride, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    if (st) { st->cpu_wall_s = t.seconds(); st->gpu_s = 0; st->cpu_submit_ns = 0; }
  });
}

azk_status azk_keccakf_plan_permute_resident(azk_keccakf_plan* p, const void* din, uint64_t in_off, void* dout, uint64_t out_off, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && din && dout);
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    keccakf_run(p, static_cast<const uint8_t*>(din) + in_off, static_cast<uint8_t*>(dout) + out_off, st, t);
  });
}

azk_status azk_keccakf_plan_clear(azk_keccakf_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaMemsetAsync(p->in.p, 0, p->in.bytes, p->s));
    AZK_CU(cudaMemsetAsync(p->out.p, 0, p->out.bytes, p->s));
    sync_stream(p->s);
  });
}
void azk_keccakf_plan_destroy(azk_keccakf_plan* p) { delete p; }

// ---- SHA3 / Keccak-256 batch ----
azk_status azk_hash_plan_create(azk_ctx* ctx, uint64_t count, uint64_t stride, uint64_t length, uint64_t out_stride, uint32_t suffix,
                                uint32_t threads, azk_hash_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // SHA3FixedOneBlockHashPlan.init (SHA3BatchHasher.swift:96-118)
    require(length <= 136, AZK_ERR_UNSUPPORTED_ONE_BLOCK_LENGTH,
            "Fixed-rate SHA3/Keccak path supports at most 136 bytes, got " + std::to_string(length) + ".");
    layout(count > 0 && stride >= length && out_stride >= 32 && count <= 0xFFFFFFFFull && stride <= 0xFFFFFFFFull && out_stride <= 0xFFFFFFFFull);
    require(suffix == 0x06 || suffix == 0x01, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "domain suffix must be 0x06 (SHA3) or 0x01 (Keccak)");
    require(threads == 0 || threads == 64 || threads == 128 || threads == 256, AZK_ERR_INVALID_KERNEL_CONFIGURATION,
            "threads per block must be 64, 128 or 256");
    AZK_CU(cudaSetDevice(ctx->device));
    auto p = std::make_unique<azk_hash_plan>();
    p->ctx = ctx;
    p->count = count;
    p->stride = stride;
    p->length = length;
    p->out_stride = out_stride;
    p->suffix = suffix;
    p->threads = threads;
    p->in.alloc(count * stride, "SHA3.Input");
    p->out.alloc(count * out_stride, "SHA3.Output");
    p->s = new_stream();
    *out = p.release();
  });
}

azk_status azk_hash_plan_hash(azk_hash_plan* p, const void* msgs, void* digests, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && digests && (msgs || p->count * p->stride == 0));
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    if (p->count * p->stride) AZK_CU(cudaMemcpyAsync(p->in.p, msgs, p->count * p->stride, cudaMemcpyHostToDevice, p->s));
    AZK_CU(launch_hash_batch(p->in.as<uint8_t>(), p->stride, (uint32_t)p->length, p->suffix, p->out.as<uint8_t>(), p->out_stride, p->count,
                             p->threads, p->s));
    uint64_t sub = t.ns();
    AZK_CU(cudaMemcpyAsync(digests, p->out.p, p->count * p->out_stride, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, sub, 0);
  });
}

azk_status azk_hash_plan_hash_resident(azk_hash_plan* p, const void* din, uint64_t in_off, void* dout, uint64_t out_off, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && din && dout);
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    GpuTimer g(p->s);
    AZK_CU(launch_hash_batch(static_cast<const uint8_t*>(din) + in_off, p->stride, (uint32_t)p->length, p->suffix,
                             static_cast<uint8_t*>(dout) + out_off, p->out_stride, p->count, p->threads, p->s));
    uint64_t sub = t.ns();
    g.stop();
    fill_stats(st, t, sub, g.seconds());
  });
}

azk_status azk_hash_plan_clear(azk_hash_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaMemsetAsync(p->in.p, 0, p->in.bytes, p->s));
    AZK_CU(cudaMemsetAsync(p->out.p, 0, p->out.bytes, p->s));
    sync_stream(p->s);
  });
}
void azk_hash_plan_destroy(azk_hash_plan* p) { delete p; }

// ---- Merkle (raw leaves) ----
azk_status azk_merkle_plan_create(azk_ctx* ctx, uint64_t count, uint64_t stride, uint64_t length, uint32_t treelet_log, azk_merkle_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // SHA3RawLeavesMerkleCommitPlan.init (MerkleCommitter.swift:552-579)
    require(count > 0 && is_pow2(count), AZK_ERR_INVALID_LEAF_COUNT, "Leaf count must be a non-zero power of two, got " + std::to_string(count) + ".");
    require(length <= 136, AZK_ERR_UNSUPPORTED_ONE_BLOCK_LENGTH,
            "Fixed-rate SHA3/Keccak path supports at most 136 bytes, got " + std::to_string(length) + ".");
    layout(stride >= length && count <= 0xFFFFFFFFull && stride <= 0xFFFFFFFFull);
    require(treelet_log <= 13, AZK_ERR_INVALID_KERNEL_CONFIGURATION, "treelet_log must be in 0...13");
    AZK_CU(cudaSetDevice(ctx->device));
    auto p = std::make_unique<azk_merkle_plan>();
    p->ctx = ctx;
    p->count = count;
    p->stride = stride;
    p->length = length;
    p->logn = ilog2(count);
    // default depth: the tuned table for one raw-leaf tree of this size
    uint32_t tl = treelet_log ? treelet_log : (p->logn < 32 && kTuned_merkle_raw64[p->logn] ? kTuned_merkle_raw64[p->logn] : 12);
    if (tl > p->logn) tl = p->logn;
    if (tl == 0 && p->logn > 0) tl = 1;
    p->tile_log = tl;
    p->threads = treelet_log ? 256 : (p->logn < 32 && kTunedThreads_merkle_raw64[p->logn] ? kTunedThreads_merkle_raw64[p->logn] : 256);
    p->leaves.alloc(count * stride, "Merkle.Leaves");
    p->leaf_digests.alloc(count * 32, "Merkle.LeafDigests");
    p->inner.alloc((count > 1 ? count - 1 : 1) * 32, "Merkle.Inner");
    uint64_t ncnt = tree_counter_count(p->logn, tl);
    p->counters.alloc(ncnt * 4, "Merkle.Counters");
    p->root.alloc(32, "Merkle.Root");
    p->job.alloc(sizeof(TreeJob), "Merkle.Job");
    p->s = new_stream();
    AZK_CU(cudaMemsetAsync(p->counters.p, 0, ncnt * 4, p->s));
    uint64_t tiles = 1ull << (p->logn - tl);
    p->h_work.resize(tiles);
    for (uint64_t i = 0; i < tiles; i++) p->h_work[i] = make_uint2(0, (uint32_t)i);
    p->work.alloc(tiles * sizeof(uint2), "Merkle.Work");
    AZK_CU(cudaMemcpyAsync(p->work.p, p->h_work.data(), tiles * sizeof(uint2), cudaMemcpyHostToDevice, p->s));
    TreeJob& j = p->h_job;
    j.logn = p->logn;
    j.kind = kLeafRaw;
    j.tile_log = tl;
    j.group_log = tl ? tl : 1;
    j.stride = stride;
    j.len = (uint32_t)length;
    j.suffix = 0x06;
    j.leaf_digests = p->leaf_digests.as<uint64_t>();
    j.inner = p->inner.as<uint64_t>();
    j.counters = p->counters.as<uint32_t>();
    j.root_out = p->root.as<uint64_t>();
    j.root_action = kRootNone;
    sync_stream(p->s);
    *out = p.release();
  });
}

static void merkle_commit_dev(azk_merkle_plan* p, const uint8_t* dleaves, uint8_t* root_out, azk_stats* st, const Timer& t) {
  p->h_job.raw = dleaves;
  p->h_job.aligned8 = (((uintptr_t)dleaves & 7) == 0 && (p->stride & 7) == 0) ? 1 : 0;
  AZK_CU(cudaMemcpyAsync(p->job.p, &p->h_job, sizeof(TreeJob), cudaMemcpyHostToDevice, p->s));
  GpuTimer g(p->s);
  AZK_CU(launch_tree_jobs(p->job.as<TreeJob>(), p->work.as<uint2>(), (uint32_t)p->h_work.size(), p->tile_log, kLeafRaw, p->threads, p->s));
  uint64_t sub = t.ns();
  g.stop();
  AZK_CU(cudaMemcpyAsync(root_out, p->root.p, 32, cudaMemcpyDeviceToHost, p->s));
  sync_stream(p->s);
  p->committed = true;
  fill_stats(st, t, sub, g.seconds());
}

azk_status azk_merkle_plan_commit(azk_merkle_plan* p, const void* leaves, uint8_t root[32], azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && root && (leaves || p->count * p->stride == 0));
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    if (p->count * p->stride) AZK_CU(cudaMemcpyAsync(p->leaves.p, leaves, p->count * p->stride, cudaMemcpyHostToDevice, p->s));
    merkle_commit_dev(p, p->leaves.as<uint8_t>(), root, st, t);
  });
}

azk_status azk_merkle_plan_commit_resident(azk_merkle_plan* p, const void* dleaves, uint64_t off, uint8_t root[32], azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && root && dleaves);
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    merkle_commit_dev(p, static_cast<const uint8_t*>(dleaves) + off, root, st, t);
  });
}

static void merkle_gather(azk_merkle_plan* p, const uint64_t* idx, uint64_t n, uint8_t* out) {
  if (p->logn == 0 || n == 0) return;
  p->idx.alloc(n * 8, "Merkle.OpenIndices");
  p->paths.alloc(n * p->logn * 32, "Merkle.OpenPaths");
  AZK_CU(cudaMemcpyAsync(p->idx.p, idx, n * 8, cudaMemcpyHostToDevice, p->s));
  AZK_CU(launch_gather_openings(p->job.as<TreeJob>(), p->idx.as<uint64_t>(), (uint32_t)n, p->paths.as<uint64_t>(), p->s));
  AZK_CU(cudaMemcpyAsync(out, p->paths.p, n * p->logn * 32, cudaMemcpyDeviceToHost, p->s));
  sync_stream(p->s);
}

azk_status azk_merkle_plan_open(azk_merkle_plan* p, const void* leaves, uint64_t index, uint8_t* leaf_out, uint8_t* sib_out, uint8_t root[32],
                                azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && root && (leaves || p->count * p->stride == 0));
    layout(index < p->count);
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    if (p->count * p->stride) AZK_CU(cudaMemcpyAsync(p->leaves.p, leaves, p->count * p->stride, cudaMemcpyHostToDevice, p->s));
    merkle_commit_dev(p, p->leaves.as<uint8_t>(), root, nullptr, t);
    merkle_gather(p, &index, 1, sib_out);
    if (leaf_out && p->length) std::memcpy(leaf_out, static_cast<const uint8_t*>(leaves) + index * p->stride, p->length);
    fill_stats(st, t, 0, 0);
  });
}

azk_status azk_merkle_plan_open_resident(azk_merkle_plan* p, const uint64_t* idx, uint64_t n, uint8_t* sib_out, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && (idx || !n) && (sib_out || !n));
    std::lock_guard<std::mutex> lk(p->mu);
    layout(p->committed, "open_resident needs a committed tree");
    for (uint64_t k = 0; k < n; k++) layout(idx[k] < p->count);
    Timer t;
    merkle_gather(p, idx, n, sib_out);
    fill_stats(st, t, 0, 0);
  });
}

azk_status azk_merkle_plan_info(azk_merkle_plan* p, uint32_t* depth, uint32_t* treelet_leaves) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    if (depth) *depth = p->logn;
    if (treelet_leaves) *treelet_leaves = 1u << p->tile_log;
  });
}

azk_status azk_merkle_plan_clear(azk_merkle_plan* p) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p != nullptr);
    std::lock_guard<std::mutex> lk(p->mu);
    for (DevBuf* b : {&p->leaves, &p->leaf_digests, &p->inner, &p->root})
      AZK_CU(cudaMemsetAsync(b->p, 0, b->bytes, p->s));
    sync_stream(p->s);
    p->committed = false;
  });
}
void azk_merkle_plan_destroy(azk_merkle_plan* p) { delete p; }

azk_status azk_merkle_commit_prehashed(azk_ctx* ctx, const void* digests, uint64_t bytes, uint8_t root[32], azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && digests && root);
    // SHA3MerkleCommitter.commitPrehashedLeaves (MerkleCommitter.swift:225-233)
    layout(bytes >= 32 && bytes % 32 == 0);
    uint64_t count = bytes / 32;
    require(is_pow2(count), AZK_ERR_INVALID_LEAF_COUNT, "Leaf count must be a non-zero power of two, got " + std::to_string(count) + ".");
    layout(count <= 0xFFFFFFFFull);
    AZK_CU(cudaSetDevice(ctx->device));
    Timer t;
    uint32_t logn = ilog2(count);
    uint32_t tl = std::min<uint32_t>(10, logn);
    if (tl == 0 && logn) tl = 1;
    DevBuf d(bytes, "Merkle.Prehashed"), inner((count > 1 ? count - 1 : 1) * 32, "Merkle.Inner"), r(32, "Merkle.Root"),
        cnt(tree_counter_count(logn, tl) * 4, "Merkle.Counters"), jb(sizeof(TreeJob), "Merkle.Job");
    uint64_t tiles = 1ull << (logn - tl);
    std::vector<uint2> w(tiles);
    for (uint64_t i = 0; i < tiles; i++) w[i] = make_uint2(0, (uint32_t)i);
    DevBuf dw(tiles * sizeof(uint2), "Merkle.Work");
    cudaStream_t s = ctx->stream;
    TreeJob j{};
    j.logn = logn;
    j.kind = kLeafDigest;
    j.tile_log = tl;
    j.group_log = tl ? tl : 1;
    j.raw = d.as<uint8_t>();
    j.inner = inner.as<uint64_t>();
    j.counters = cnt.as<uint32_t>();
    j.root_out = r.as<uint64_t>();
    AZK_CU(cudaMemcpyAsync(d.p, digests, bytes, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
    AZK_CU(cudaMemcpyAsync(dw.p, w.data(), tiles * sizeof(uint2), cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemcpyAsync(jb.p, &j, sizeof(TreeJob), cudaMemcpyHostToDevice, s));
    GpuTimer g(s);
    AZK_CU(launch_tree_jobs(jb.as<TreeJob>(), dw.as<uint2>(), (uint32_t)tiles, tl, kLeafDigest, 256, s));
    g.stop();
    AZK_CU(cudaMemcpyAsync(root, r.p, 32, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
    fill_stats(st, t, 0, g.seconds());
  });
}

// ---- SHA3PrehashedLeavesMerkleCommitPlan (MerkleCommitter.swift:314-524) ----
azk_status azk_merkle_prehashed_plan_create(azk_ctx* ctx, uint64_t leaf_count, azk_merkle_prehashed_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    // init (:330-334): a non-zero power of two that fits 32 bits
    require(is_pow2(leaf_count), AZK_ERR_INVALID_LEAF_COUNT, "Leaf count must be a non-zero power of two, got " + std::to_string(leaf_count) + ".");
    layout(leaf_count <= 0xFFFFFFFFull);
    AZK_CU(cudaSetDevice(ctx->device));
    auto p = std::make_unique<azk_merkle_prehashed_plan>();
    p->ctx = ctx;
    p->count = leaf_count;
    p->logn = ilog2(leaf_count);
    p->tile_log = std::min<uint32_t>(10, p->logn);
    if (p->tile_log == 0 && p->logn) p->tile_log = 1;
    p->s = new_stream();
    p->staging.alloc(32 * leaf_count, "Merkle.PrehashedPlanLeaves");
    p->inner.alloc((leaf_count > 1 ? leaf_count - 1 : 1) * 32, "Merkle.PrehashedPlanInner");
    p->counters.alloc(tree_counter_count(p->logn, p->tile_log) * 4, "Merkle.PrehashedPlanCounters");
    p->root.alloc(32, "Merkle.PrehashedPlanRoot");
    p->job.alloc(sizeof(TreeJob), "Merkle.PrehashedPlanJob");
    const uint64_t tiles = 1ull << (p->logn - p->tile_log);
    std::vector<uint2> w(tiles);
    for (uint64_t i = 0; i < tiles; i++) w[i] = make_uint2(0, (uint32_t)i);
    p->work.alloc(tiles * sizeof(uint2), "Merkle.PrehashedPlanWork");
    TreeJob& j = p->h_job;
    j.logn = p->logn;
    j.kind = kLeafDigest;
    j.tile_log = p->tile_log;
    j.group_log = p->tile_log ? p->tile_log : 1;
    j.inner = p->inner.as<uint64_t>();
    j.counters = p->counters.as<uint32_t>();
    j.root_out = p->root.as<uint64_t>();
    AZK_CU(cudaMemsetAsync(p->counters.p, 0, p->counters.bytes, p->s));
    AZK_CU(cudaMemcpyAsync(p->work.p, w.data(), tiles * sizeof(uint2), cudaMemcpyHostToDevice, p->s));
    sync_stream(p->s);
    *out = p.release();
  });
}

static void prehashed_commit(azk_merkle_prehashed_plan* p, const uint8_t* leaves, uint8_t root[32], azk_stats* st, const Timer& t) {
  p->h_job.raw = leaves;
  AZK_CU(cudaMemcpyAsync(p->job.p, &p->h_job, sizeof(TreeJob), cudaMemcpyHostToDevice, p->s));
  GpuTimer g(p->s);
  AZK_CU(launch_tree_jobs(p->job.as<TreeJob>(), p->work.as<uint2>(), (uint32_t)(1ull << (p->logn - p->tile_log)), p->tile_log, kLeafDigest, 256, p->s));
  g.stop();
  AZK_CU(cudaMemcpyAsync(root, p->root.p, 32, cudaMemcpyDeviceToHost, p->s));
  sync_stream(p->s);
  fill_stats(st, t, 0, g.seconds());
}

azk_status azk_merkle_prehashed_plan_commit(azk_merkle_prehashed_plan* p, const void* host_digests, uint8_t root_out[32], azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && host_digests && root_out);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    AZK_CU(cudaMemcpyAsync(p->staging.p, host_digests, 32 * p->count, cudaMemcpyHostToDevice, p->s));
    prehashed_commit(p, p->staging.as<uint8_t>(), root_out, st, t);
  });
}

azk_status azk_merkle_prehashed_plan_commit_resident(azk_merkle_prehashed_plan* p, const void* dev_digests, uint64_t offset, uint8_t root_out[32],
                                                     azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && root_out);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    require_device_range(dev_digests, offset, 32 * p->count);
    // the digests are read as 16-byte vectors
    layout((reinterpret_cast<uintptr_t>(dev_digests) + offset) % 16 == 0, "resident digests must start on a 16-byte boundary");
    Timer t;
    prehashed_commit(p, static_cast<const uint8_t*>(dev_digests) + offset, root_out, st, t);
  });
}

void azk_merkle_prehashed_plan_destroy(azk_merkle_prehashed_plan* p) { delete p; }

// ---- circle domain ----
azk_status azk_circle_domain_points(azk_ctx* ctx, uint32_t logn, uint32_t* xy) {
  return guarded(ctx, [&] {
    layout(ctx && xy && logn >= 1 && logn <= 26);
    AZK_CU(cudaSetDevice(ctx->device));
    uint64_t n = 1ull << logn;
    DevBuf d(8 * n, "CircleDomain.Points");
    AZK_CU(launch_domain_points(logn, d.as<uint32_t>(), ctx->stream));
    AZK_CU(cudaMemcpyAsync(xy, d.p, 8 * n, cudaMemcpyDeviceToHost, ctx->stream));
    sync_stream(ctx->stream);
  });
}

azk_status azk_circle_fft_twiddles(azk_ctx* ctx, uint32_t logn, uint32_t* out) {
  return guarded(ctx, [&] {
    layout(ctx && out);
    AZK_CU(cudaSetDevice(ctx->device));
    const auto& d = domain_tables(ctx, logn);
    uint64_t n = 1ull << logn;
    AZK_CU(cudaMemcpy(out, d.tw, 4 * (n - 1), cudaMemcpyDeviceToHost));
  });
}

azk_status azk_circle_inverse_layers(azk_ctx* ctx, uint32_t logn, uint32_t rounds, uint32_t* out) {
  return guarded(ctx, [&] {
    layout(ctx && out && rounds >= 1 && rounds <= logn);
    AZK_CU(cudaSetDevice(ctx->device));
    const auto& d = domain_tables(ctx, logn);
    uint64_t n = 1ull << logn, total = n - (n >> rounds);
    AZK_CU(cudaMemcpy(out, d.inv, 4 * total, cudaMemcpyDeviceToHost));
  });
}

// ---- codeword ----
azk_status azk_codeword_plan_create(azk_ctx* ctx, uint32_t logn, azk_codeword_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && logn >= 1 && logn <= 26);
    AZK_CU(cudaSetDevice(ctx->device));
    const auto& d = domain_tables(ctx, logn);
    auto p = std::make_unique<azk_codeword_plan>();
    p->ctx = ctx;
    p->logn = logn;
    uint64_t n = 1ull << logn;
    p->coeff.alloc(16 * n, "CircleCodeword.Coefficients");
    p->out.alloc(16 * n, "CircleCodeword.Output");
    p->s = new_stream();
    FftJob j{logn, 0, p->coeff.as<uint4>(), p->out.as<uint4>(), d.tw};
    p->fft.build({j});
    p->fft.upload(p->s);
    sync_stream(p->s);
    *out = p.release();
  });
}

static void codeword_run(azk_codeword_plan* p, const uint4* din, uint4* dout, azk_stats* st, const Timer& t) {
  const auto& d = domain_tables(p->ctx, p->logn);
  FftJob j{p->logn, 0, din, dout, d.tw};
  bool same = din == p->coeff.as<uint4>() && dout == p->out.as<uint4>();
  if (!same) {
    p->fft.build({j});
    p->fft.upload(p->s);
  }
  GpuTimer g(p->s);
  p->fft.launch_all(p->s);
  uint64_t sub = t.ns();
  g.stop();
  double gs = g.seconds();
  if (!same) {
    FftJob back{p->logn, 0, p->coeff.as<uint4>(), p->out.as<uint4>(), d.tw};
    p->fft.build({back});
    p->fft.upload(p->s);
  }
  fill_stats(st, t, sub, gs);
}

azk_status azk_codeword_plan_execute(azk_codeword_plan* p, const uint32_t* coeffs, uint64_t count, uint32_t* codeword, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && codeword && (coeffs || !count));
    uint64_t n = 1ull << p->logn;
    layout(count <= n);
    layout(all_canonical(coeffs, 4 * count));
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    if (count) AZK_CU(cudaMemcpyAsync(p->coeff.p, coeffs, 16 * count, cudaMemcpyHostToDevice, p->s));
    if (count < n) AZK_CU(cudaMemsetAsync(p->coeff.as<uint4>() + count, 0, 16 * (n - count), p->s));
    codeword_run(p, p->coeff.as<uint4>(), p->out.as<uint4>(), nullptr, t);
    AZK_CU(cudaMemcpyAsync(codeword, p->out.p, 16 * n, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
    fill_stats(st, t, 0, 0);
  });
}

// execute(polynomial:) (CircleCodeword.swift:460-475): the monomial columns become
// FFT-basis coefficients on the device (the witness plan's closed-form Chebyshev
// and line-basis kernels, domains up to 2^22), then the FFT.  Larger domains keep
// the reference's host conversion (CircleCodeword.swift:187-263).
azk_status azk_codeword_plan_execute_polynomial(azk_codeword_plan* p, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny, uint32_t* codeword,
                                                azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && codeword && (x || !nx) && (y || !ny));
    if (p->logn > 22 || nx + ny == 0) {
      std::vector<uint32_t> c = fft_basis_from_monomials(p->logn, x, nx, y, ny);
      azk_status s = azk_codeword_plan_execute(p, c.data(), c.size() / 4, codeword, st);
      if (s != AZK_OK) fail(s, azk_last_error_message(p->ctx));
      return;
    }
    const uint64_t half = (1ull << p->logn) / 2;
    layout(nx <= half && ny <= half, "each coefficient column holds at most half the domain size");
    layout(all_canonical(x, 4 * nx), "input contains a non-canonical field element");
    layout(all_canonical(y, 4 * ny), "input contains a non-canonical field element");
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    Timer t;
    if (!p->wit) {
      azk_status s = azk_witness_plan_create(p->ctx, p->logn, &p->wit);
      if (s != AZK_OK) fail(s, azk_last_error_message(p->ctx));
    }
    witness_columns_to_device(p->wit, x, nx, y, ny, p->coeff.p);
    codeword_run(p, p->coeff.as<uint4>(), p->out.as<uint4>(), st, t);
    AZK_CU(cudaMemcpyAsync(codeword, p->out.p, 16ull << p->logn, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
  });
}

azk_status azk_codeword_plan_execute_resident(azk_codeword_plan* p, const void* din, uint64_t in_off, void* dout, uint64_t out_off, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && din && dout && in_off % 16 == 0 && out_off % 16 == 0);
    std::lock_guard<std::mutex> lk(p->mu);
    AZK_CU(cudaSetDevice(p->ctx->device));
    // executeResident's buffer-length checks (CircleCodeword.swift:517-545): N
    // coefficients in, N codeword values out, the two not overlapping
    const uint64_t bytes = 16ull << p->logn;
    require_device_range(din, in_off, bytes);
    require_device_range(dout, out_off, bytes);
    layout(!ranges_overlap(din, in_off, bytes, dout, out_off, bytes), "the codeword output overlaps the coefficients");
    Timer t;
    codeword_run(p, reinterpret_cast<const uint4*>(static_cast<const uint8_t*>(din) + in_off),
                 reinterpret_cast<uint4*>(static_cast<uint8_t*>(dout) + out_off), st, t);
    sync_stream(p->s);
  });
}
void azk_codeword_plan_destroy(azk_codeword_plan* p) { delete p; }

}  // extern "C"

// ---- witness columns -> FFT basis (CircleWitnessToFFTBasisPlanV1) ----
struct azk_witness_plan {
  azk_ctx* ctx;
  std::mutex mu;
  cudaStream_t s = nullptr;
  uint32_t logn;
  uint64_t n;  // coefficient capacity = half the domain
  DevBuf fact, seg, ifact, scale, ax, ay, px, py, cx, cy, xin, yin, out, flag;
  ~azk_witness_plan() {
    if (s) cudaStreamDestroy(s);
  }
};

static void witness_run(azk_witness_plan* p, const uint4* x, uint64_t nx, const uint4* y, uint64_t ny, uint4* out, azk_stats* st, const Timer& t) {
  // canonicality of both columns (CircleWitnessFFTBasis.swift:374-385)
  AZK_CU(cudaMemsetAsync(p->flag.p, 0, 4, p->s));
  if (nx) AZK_CU(launch_check_canonical(reinterpret_cast<const uint32_t*>(x), 4 * nx, p->flag.as<uint32_t>(), p->s));
  if (ny) AZK_CU(launch_check_canonical(reinterpret_cast<const uint32_t*>(y), 4 * ny, p->flag.as<uint32_t>(), p->s));
  uint32_t bad = 0;
  AZK_CU(cudaMemcpyAsync(&bad, p->flag.p, 4, cudaMemcpyDeviceToHost, p->s));
  sync_stream(p->s);
  layout(bad == 0, "witness coefficients contain a non-canonical field element");
  GpuTimer g(p->s);
  AZK_CU(launch_witness_transform(x, nx, y, ny, p->n, p->ifact.as<uint32_t>(), p->scale.as<uint32_t>(), p->ax.as<uint4>(), p->ay.as<uint4>(),
                                  p->px.as<uint4>(), p->py.as<uint4>(), p->cx.as<uint4>(), p->cy.as<uint4>(), out, p->s));
  g.stop();
  fill_stats(st, t, 0, g.seconds());
}

static void witness_columns_to_device(azk_witness_plan* w, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny, void* dout) {
  std::lock_guard<std::mutex> lk(w->mu);
  Timer t;
  if (nx) AZK_CU(cudaMemcpyAsync(w->xin.p, x, 16 * nx, cudaMemcpyHostToDevice, w->s));
  if (ny) AZK_CU(cudaMemcpyAsync(w->yin.p, y, 16 * ny, cudaMemcpyHostToDevice, w->s));
  witness_run(w, w->xin.as<uint4>(), nx, w->yin.as<uint4>(), ny, static_cast<uint4*>(dout), nullptr, t);
  sync_stream(w->s);
}

extern "C" {

azk_status azk_witness_plan_create(azk_ctx* ctx, uint32_t log_size, azk_witness_plan** out) {
  return guarded(ctx, [&] {
    layout(ctx && out && log_size >= 1 && log_size <= 22);
    AZK_CU(cudaSetDevice(ctx->device));
    auto p = std::make_unique<azk_witness_plan>();
    p->ctx = ctx;
    p->logn = log_size;
    p->n = 1ull << (log_size - 1);
    p->s = new_stream();
    const uint64_t n = p->n;
    p->fact.alloc(4 * n, "Witness.Factorials");
    p->seg.alloc(4 * ((n + 1023) / 1024), "Witness.Segments");
    p->ifact.alloc(4 * n, "Witness.InverseFactorials");
    p->scale.alloc(4 * n, "Witness.Scale");
    for (DevBuf* b : {&p->ax, &p->ay, &p->cx, &p->cy, &p->xin, &p->yin}) b->alloc(16 * n, "Witness.Scratch");
    p->px.alloc(16 * witness_partial_values(n), "Witness.PartialSums");
    p->py.alloc(16 * witness_partial_values(n), "Witness.PartialSums");
    p->out.alloc(32 * n, "Witness.Output");
    p->flag.alloc(16, "Witness.Flag");
    AZK_CU(launch_witness_tables(n, p->fact.as<uint32_t>(), p->seg.as<uint32_t>(), p->ifact.as<uint32_t>(), p->scale.as<uint32_t>(), p->s));
    sync_stream(p->s);
    *out = p.release();
  });
}

// Host columns x, y of monomial coefficients (QM31) -> 2 * capacity interleaved
// FFT-basis coefficients [x0, y0, x1, y1, ...].
azk_status azk_witness_plan_execute(azk_witness_plan* p, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny, uint32_t* out,
                                    azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && out && (x || !nx) && (y || !ny));
    // CircleWitnessFFTBasis.swift:349-353
    layout(nx <= p->n && ny <= p->n && nx + ny > 0);
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    if (nx) AZK_CU(cudaMemcpyAsync(p->xin.p, x, 16 * nx, cudaMemcpyHostToDevice, p->s));
    if (ny) AZK_CU(cudaMemcpyAsync(p->yin.p, y, 16 * ny, cudaMemcpyHostToDevice, p->s));
    witness_run(p, p->xin.as<uint4>(), nx, p->yin.as<uint4>(), ny, p->out.as<uint4>(), st, t);
    AZK_CU(cudaMemcpyAsync(out, p->out.p, 32 * p->n, cudaMemcpyDeviceToHost, p->s));
    sync_stream(p->s);
  });
}

// executeResident (CircleWitnessFFTBasis.swift:320-428): device columns and a
// device output of 2 * capacity QM31 that must not overlap either column.
azk_status azk_witness_plan_execute_resident(azk_witness_plan* p, const void* dx, uint64_t x_off, uint64_t nx, const void* dy, uint64_t y_off, uint64_t ny,
                                             void* dout, uint64_t out_off, azk_stats* st) {
  return guarded(p ? p->ctx : nullptr, [&] {
    layout(p && dout && (dx || !nx) && (dy || !ny));
    layout(nx <= p->n && ny <= p->n && nx + ny > 0);
    layout(x_off % 16 == 0 && y_off % 16 == 0 && out_off % 16 == 0);
    const uint8_t* xb = static_cast<const uint8_t*>(dx) + x_off;
    const uint8_t* yb = static_cast<const uint8_t*>(dy) + y_off;
    uint8_t* ob = static_cast<uint8_t*>(dout) + out_off;
    const uint64_t ob_len = 32 * p->n;
    auto overlap = [&](const uint8_t* a, uint64_t alen) { return alen && a < ob + ob_len && ob < a + alen; };
    layout(!overlap(xb, 16 * nx) && !overlap(yb, 16 * ny), "the output range overlaps a witness column");
    std::lock_guard<std::mutex> lk(p->mu);
    Timer t;
    witness_run(p, reinterpret_cast<const uint4*>(xb), nx, reinterpret_cast<const uint4*>(yb), ny, reinterpret_cast<uint4*>(ob), st, t);
    sync_stream(p->s);
  });
}

void azk_witness_plan_destroy(azk_witness_plan* p) { delete p; }

// ---- folds ----
static void check_qm31(const uint32_t* v, uint64_t words) {
  layout(all_canonical(v, words));
}

azk_status azk_qm31_fold(azk_ctx* ctx, const uint32_t* ev, uint64_t n, const uint32_t* inv, const uint32_t ch[4], uint32_t* out, azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && ev && inv && ch && out);
    // QM31FRIFoldOracle.fold preconditions (QM31FRIFold.swift:16-27)
    layout(n > 1 && n % 2 == 0);
    check_qm31(ev, 4 * n);
    check_qm31(inv, 2 * n);
    check_qm31(ch, 4);
    for (uint64_t i = 0; i < n / 2; i++) layout(inv[4 * i] | inv[4 * i + 1] | inv[4 * i + 2] | inv[4 * i + 3]);
    AZK_CU(cudaSetDevice(ctx->device));
    Timer t;
    cudaStream_t s = ctx->stream;
    DevBuf de(16 * n, "QM31Fold.Input"), di(8 * n, "QM31Fold.Inverse"), dc(16, "QM31Fold.Challenge"), dout(8 * n, "QM31Fold.Output");
    AZK_CU(cudaMemcpyAsync(de.p, ev, 16 * n, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemcpyAsync(di.p, inv, 8 * n, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemcpyAsync(dc.p, ch, 16, cudaMemcpyHostToDevice, s));
    GpuTimer g(s);
    AZK_CU(launch_fold_qm31_inv(de.as<uint4>(), di.as<uint4>(), dc.as<uint32_t>(), dout.as<uint4>(), n / 2, s));
    g.stop();
    AZK_CU(cudaMemcpyAsync(out, dout.p, 8 * n, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_circle_fold_chain(azk_ctx* ctx, uint32_t logn, const uint32_t* ev, const uint32_t* ch, uint32_t rounds, uint32_t* out, azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && ev && ch && out && logn >= 1 && logn <= 26 && rounds >= 1 && rounds <= logn);
    uint64_t n = 1ull << logn;
    check_qm31(ev, 4 * n);
    check_qm31(ch, 4ull * rounds);
    AZK_CU(cudaSetDevice(ctx->device));
    const auto& d = domain_tables(ctx, logn);
    Timer t;
    cudaStream_t s = ctx->stream;
    DevBuf layers(16 * 2 * n, "CircleFold.Layers"), dch(16ull * rounds, "CircleFold.Challenges");
    AZK_CU(cudaMemcpyAsync(layers.p, ev, 16 * n, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemcpyAsync(dch.p, ch, 16ull * rounds, cudaMemcpyHostToDevice, s));
    std::vector<FoldJob> jobs;
    std::vector<uint2> work;
    for (uint32_t r = 0; r < rounds; r++) {
      FoldJob j{n >> (r + 1), layers.as<uint4>() + layer_offset(logn, r), d.inv + (r == 0 ? 0 : n - (n >> r)), dch.as<uint32_t>() + 4 * r,
                layers.as<uint4>() + layer_offset(logn, r + 1)};
      jobs.push_back(j);
    }
    DevBuf djobs(jobs.size() * sizeof(FoldJob), "CircleFold.Jobs");
    AZK_CU(cudaMemcpyAsync(djobs.p, jobs.data(), jobs.size() * sizeof(FoldJob), cudaMemcpyHostToDevice, s));
    std::vector<std::pair<uint64_t, uint64_t>> ranges;
    for (uint32_t r = 0; r < rounds; r++) {
      uint64_t chunks = (jobs[r].n_out + kFoldChunk - 1) / kFoldChunk;
      ranges.push_back({work.size(), chunks});
      for (uint64_t c = 0; c < chunks; c++) work.push_back(make_uint2(r, (uint32_t)c));
    }
    DevBuf dwork(work.size() * sizeof(uint2), "CircleFold.Work");
    AZK_CU(cudaMemcpyAsync(dwork.p, work.data(), work.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
    GpuTimer g(s);
    for (uint32_t r = 0; r < rounds; r++)
      AZK_CU(launch_fold_jobs(djobs.as<FoldJob>(), dwork.as<uint2>() + ranges[r].first, (uint32_t)ranges[r].second, s));
    g.stop();
    AZK_CU(cudaMemcpyAsync(out, layers.as<uint4>() + layer_offset(logn, rounds), 16 * (n >> rounds), cudaMemcpyDeviceToHost, s));
    sync_stream(s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_qm31_merkle_fold_chain(azk_ctx* ctx, const uint32_t* ev, uint64_t n, const uint32_t* inv, uint32_t rounds, uint32_t* final_out,
                                      uint8_t* commitments_out, uint32_t* ch_out, azk_stats* st) {
  return guarded(ctx, [&] {
    layout(ctx && ev && inv && final_out && rounds >= 1);
    // QM31FRIMerkleFoldChainOracle.commitAndFold preconditions (QM31FRIFold.swift:168-193)
    layout(n > 1 && is_pow2(n) && (n >> rounds) >= 1 && rounds <= ilog2(n));
    check_qm31(ev, 4 * n);
    uint64_t inv_total = n - (n >> rounds);
    check_qm31(inv, 4 * inv_total);
    for (uint64_t i = 0; i < inv_total; i++) layout(inv[4 * i] | inv[4 * i + 1] | inv[4 * i + 2] | inv[4 * i + 3]);
    AZK_CU(cudaSetDevice(ctx->device));
    Timer t;
    cudaStream_t s = ctx->stream;
    uint32_t logn = ilog2(n);
    DevBuf layers(16 * 2 * n, "QM31Chain.Layers"), dinv(16 * inv_total + 16, "QM31Chain.Inverse"), dch(16ull * rounds, "QM31Chain.Challenges"),
        dcm(32ull * rounds, "QM31Chain.Commitments"), tr(sizeof(Transcript), "QM31Chain.Transcript"), inner(32 * n, "QM31Chain.Inner"),
        cnt(tree_counter_count(logn, 10) * 4, "QM31Chain.Counters"), jobs(sizeof(TreeJob) * rounds, "QM31Chain.Jobs");
    AZK_CU(cudaMemcpyAsync(layers.p, ev, 16 * n, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemcpyAsync(dinv.p, inv, 16 * inv_total, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemsetAsync(cnt.p, 0, cnt.bytes, s));
    std::vector<TreeJob> hj(rounds);
    std::vector<uint2> work;
    std::vector<std::pair<uint64_t, uint64_t>> ranges;
    for (uint32_t r = 0; r < rounds; r++) {
      uint32_t lg = logn - r;
      uint32_t tl = std::min<uint32_t>(10, lg);
      if (tl == 0 && lg) tl = 1;
      TreeJob& j = hj[r];
      j = TreeJob{};
      j.logn = lg;
      j.kind = kLeafQM31;
      j.tile_log = tl;
      j.group_log = tl ? tl : 1;
      j.layer = layers.as<uint4>() + layer_offset(logn, r);
      j.inner = inner.as<uint64_t>();
      j.counters = cnt.as<uint32_t>();
      j.root_action = kRootQM31Round;
      j.round = r;
      j.frame_in_count = n >> r;
      j.transcript = tr.as<Transcript>();
      j.challenge_out = dch.as<uint32_t>() + 4 * r;
      j.root_out = dcm.as<uint64_t>() + 4 * r;
      uint64_t tiles = 1ull << (lg - tl);
      ranges.push_back({work.size(), tiles});
      for (uint64_t k = 0; k < tiles; k++) work.push_back(make_uint2(r, (uint32_t)k));
    }
    DevBuf dwork(work.size() * sizeof(uint2), "QM31Chain.Work");
    AZK_CU(cudaMemcpyAsync(jobs.p, hj.data(), sizeof(TreeJob) * rounds, cudaMemcpyHostToDevice, s));
    AZK_CU(cudaMemcpyAsync(dwork.p, work.data(), work.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
    GpuTimer g(s);
    AZK_CU(launch_qm31_transcript_prefix(tr.as<Transcript>(), n, rounds, s));
    uint64_t inv_off = 0;
    for (uint32_t r = 0; r < rounds; r++) {
      AZK_CU(launch_tree_jobs(jobs.as<TreeJob>(), dwork.as<uint2>() + ranges[r].first, (uint32_t)ranges[r].second, hj[r].tile_log, kLeafQM31, 256, s));
      uint64_t m = n >> (r + 1);
      AZK_CU(launch_fold_qm31_inv(layers.as<uint4>() + layer_offset(logn, r), dinv.as<uint4>() + inv_off, dch.as<uint32_t>() + 4 * r,
                                  layers.as<uint4>() + layer_offset(logn, r + 1), m, s));
      inv_off += m;
    }
    g.stop();
    AZK_CU(cudaMemcpyAsync(final_out, layers.as<uint4>() + layer_offset(logn, rounds), 16 * (n >> rounds), cudaMemcpyDeviceToHost, s));
    if (commitments_out) AZK_CU(cudaMemcpyAsync(commitments_out, dcm.p, 32ull * rounds, cudaMemcpyDeviceToHost, s));
    if (ch_out) AZK_CU(cudaMemcpyAsync(ch_out, dch.p, 16ull * rounds, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
    fill_stats(st, t, 0, g.seconds());
  });
}

azk_status azk_qm31_transcript_challenges(azk_ctx* ctx, uint64_t input_count, const uint8_t* commitments, uint32_t rounds, uint32_t* ch_out) {
  return guarded(ctx, [&] {
    layout(ctx && commitments && ch_out && rounds >= 1);
    layout(input_count > 1);
    uint64_t c = input_count;
    for (uint32_t r = 0; r < rounds; r++) {
      layout(c > 1 && c % 2 == 0);
      c /= 2;
    }
    AZK_CU(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    DevBuf tr(sizeof(Transcript), "Transcript"), roots(32ull * rounds, "Roots"), dch(16ull * rounds, "Challenges");
    AZK_CU(cudaMemcpyAsync(roots.p, commitments, 32ull * rounds, cudaMemcpyHostToDevice, s));
    AZK_CU(launch_qm31_transcript_prefix(tr.as<Transcript>(), input_count, rounds, s));
    AZK_CU(launch_transcript_rounds_given(tr.as<Transcript>(), kRootQM31Round, roots.as<uint64_t>(), rounds, input_count, dch.as<uint32_t>(), s));
    AZK_CU(cudaMemcpyAsync(ch_out, dch.p, 16ull * rounds, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
  });
}

azk_status azk_probe_int_issue(azk_ctx* ctx, double* ops_per_second) {
  return guarded(ctx, [&] {
    layout(ctx && ops_per_second);
    AZK_CU(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    DevBuf sink(16, "Probe.Sink");
    double ops = 0;
    AZK_CU(launch_int_issue_probe(ctx->sm_count, s, sink.as<uint32_t>(), &ops, nullptr));  // warm-up
    sync_stream(s);
    double best = 0;
    for (int rep = 0; rep < 5; rep++) {
      GpuTimer g(s);
      AZK_CU(launch_int_issue_probe(ctx->sm_count, s, sink.as<uint32_t>(), &ops, nullptr));
      g.stop();
      double sec = g.seconds();
      if (sec > 0) best = std::max(best, ops / sec);
    }
    *ops_per_second = best;
  });
}

azk_status azk_check_canonical(azk_ctx* ctx, const void* dwords, uint64_t nwords, uint32_t* flag_out) {
  return guarded(ctx, [&] {
    layout(ctx && dwords && flag_out);
    AZK_CU(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    DevBuf f(4, "Canonical.Flag");
    AZK_CU(cudaMemsetAsync(f.p, 0, 4, s));
    AZK_CU(launch_check_canonical(static_cast<const uint32_t*>(dwords), nwords, f.as<uint32_t>(), s));
    AZK_CU(cudaMemcpyAsync(flag_out, f.p, 4, cudaMemcpyDeviceToHost, s));
    sync_stream(s);
  });
}

}  // extern "C"
