// Host-side runtime shared by the C-ABI translation units: context, error
// handling, device buffers, domain-table cache and the work-list builders.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/azk_cuda.h"
#include "azk_internal.h"

struct azk_ctx {
  int device = 0;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  uint64_t total_mem = 0;
  cudaStream_t stream = nullptr;
  std::mutex mu;
  std::string last_error;
  struct Domain {
    uint32_t* tw = nullptr;  // N - 1 stage twiddles, then (at tw + N) the same doubled
    uint32_t* inv = nullptr;
  };
  std::map<uint32_t, Domain> domains;
};

namespace azk {

struct Error {
  azk_status code;
  std::string msg;
};

[[noreturn]] inline void fail(azk_status code, const std::string& msg) { throw Error{code, msg}; }
inline void require(bool ok, azk_status code, const std::string& msg) {
  if (!ok) fail(code, msg);
}
inline void layout(bool ok, const char* what = "The provided input bytes do not match the declared count/stride/length layout.") {
  if (!ok) fail(AZK_ERR_INVALID_INPUT_LAYOUT, what);
}
// Whether all `n` words are canonical M31 values (below 2^31 - 1): one
// branch-free pass that the host compiler vectorises (a 4 MiB table in about
// 0.1 ms, against about 1 ms for a compare-and-branch per word).
inline bool all_canonical(const uint32_t* w, uint64_t n) {
  uint32_t bad = 0;
  for (uint64_t i = 0; i < n; i++) bad |= (uint32_t)(w[i] >= 2147483647u);
  return bad == 0;
}

#define AZK_CU(expr)                                                                                   \
  do {                                                                                                 \
    cudaError_t azk_e_ = (expr);                                                                       \
    if (azk_e_ != cudaSuccess)                                                                         \
      ::azk::fail(AZK_ERR_COMMAND_EXECUTION_FAILED, std::string(#expr) + ": " + cudaGetErrorString(azk_e_)); \
  } while (0)

void set_error(const azk_ctx* ctx, const std::string& msg);

template <class F>
azk_status guarded(const azk_ctx* ctx, F&& f) {
  try {
    f();
    return AZK_OK;
  } catch (const Error& e) {
    set_error(ctx, e.msg);
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error(ctx, "host allocation failed");
    return AZK_ERR_FAILED_TO_CREATE_BUFFER;
  } catch (const std::exception& e) {
    set_error(ctx, e.what());
    return AZK_ERR_COMMAND_EXECUTION_FAILED;
  }
}

inline bool is_pow2(uint64_t v) { return v && !(v & (v - 1)); }
inline uint32_t ilog2(uint64_t v) {
  uint32_t r = 0;
  while (v > 1) { v >>= 1; r++; }
  return r;
}
inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

// Owning device allocation.
struct DevBuf {
  void* p = nullptr;
  uint64_t bytes = 0;
  DevBuf() = default;
  explicit DevBuf(uint64_t n, const char* label = "buffer") { alloc(n, label); }
  void alloc(uint64_t n, const char* label = "buffer") {
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      fail(AZK_ERR_FAILED_TO_CREATE_BUFFER, std::string("Failed to create device buffer '") + label + "' of length " + std::to_string(n));
    }
    bytes = n;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      bytes = o.bytes;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

// Bump allocator over one device allocation (the reference's ResidencyArena,
// Planner/ResidencyArena.swift:36-92: 256-byte aligned slices).
struct Arena {
  DevBuf buf;
  uint64_t used = 0;
  std::vector<std::pair<uint64_t, uint64_t>> plan;  // (offset, bytes) reservations before alloc
  uint64_t reserve(uint64_t bytes) {
    uint64_t off = align_up(used, 256);
    used = off + (bytes ? bytes : 16);
    return off;
  }
  void commit(const char* label) { buf.alloc(used, label); }
  template <class T>
  T* at(uint64_t off) const { return reinterpret_cast<T*>(reinterpret_cast<uint8_t*>(buf.p) + off); }
};

struct Timer {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double seconds() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
  uint64_t ns() const { return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count(); }
};

// Wait for an event by polling it: a short spin, then sleeps growing from 20 to
// 160 us, so a waiting thread takes little of a host core (the server's workers
// share the host's cores with each other and with the threads that submit work).
// Not cudaEventSynchronize on a blocking-sync event, which sleeps until the
// driver's completion interrupt: with the server's 32 workers waiting that way at
// once, the device stopped starting work for 40-80 ms about every 2 s.
inline void wait_event(cudaEvent_t e) {
  for (int k = 0;; k++) {
    const cudaError_t q = cudaEventQuery(e);
    if (q == cudaSuccess) return;
    if (q != cudaErrorNotReady) AZK_CU(q);
    if (k < 8) continue;
    std::this_thread::sleep_for(std::chrono::microseconds(k < 24 ? 20 : k < 48 ? 50 : 160));
  }
}

// Wait for everything queued on a stream (wait_event on a per-thread event).
inline void sync_stream(cudaStream_t s) {
  struct Ev {
    cudaEvent_t e = nullptr;
    int dev = -1;
    ~Ev() {
      if (e) cudaEventDestroy(e);
    }
  };
  thread_local Ev ev;
  int dev = 0;
  AZK_CU(cudaGetDevice(&dev));
  if (!ev.e || ev.dev != dev) {
    if (ev.e) cudaEventDestroy(ev.e);
    ev.e = nullptr;
    AZK_CU(cudaEventCreateWithFlags(&ev.e, cudaEventDisableTiming));
    ev.dev = dev;
  }
  AZK_CU(cudaEventRecord(ev.e, s));
  wait_event(ev.e);
}

// CUDA events around a region of one stream.
struct GpuTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  bool owns = true;
  explicit GpuTimer(cudaStream_t st) : s(st) {
    AZK_CU(cudaEventCreate(&a));
    AZK_CU(cudaEventCreate(&b));
    AZK_CU(cudaEventRecord(a, s));
  }
  // With events the caller keeps (nothing created or destroyed per region).
  GpuTimer(cudaStream_t st, cudaEvent_t ea, cudaEvent_t eb) : a(ea), b(eb), s(st), owns(false) { AZK_CU(cudaEventRecord(a, s)); }
  void stop() { AZK_CU(cudaEventRecord(b, s)); }
  double seconds() {
    float ms = 0;
    wait_event(b);
    AZK_CU(cudaEventElapsedTime(&ms, a, b));
    return ms / 1000.0;
  }
  ~GpuTimer() {
    if (!owns) return;
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Page-locked host memory kept for the owner's lifetime: small uploads and
// readbacks go through it rather than through pageable memory, which the driver
// stages through buffers shared by every thread of the process.
struct HostPinned {
  void* p = nullptr;
  size_t n = 0;
  HostPinned() = default;
  HostPinned(const HostPinned&) = delete;
  HostPinned& operator=(const HostPinned&) = delete;
  void* ensure(size_t bytes) {
    if (bytes > n) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      n = 0;
      AZK_CU(cudaHostAlloc(&p, bytes, cudaHostAllocDefault));
      n = bytes;
    }
    return p;
  }
  ~HostPinned() {
    if (p) cudaFreeHost(p);
  }
};

inline void fill_stats(azk_stats* st, const Timer& t, uint64_t submit_ns, double gpu_s) {
  if (!st) return;
  st->cpu_wall_s = t.seconds();
  st->gpu_s = gpu_s;
  st->cpu_submit_ns = submit_ns;
}

// Resident entry points take (device pointer, byte offset) pairs.  This checks
// that [p + off, p + off + bytes) lies inside the one device allocation containing
// p + off (the reference's buffer-length check, e.g. QM31FRIFold.swift:1236-1244),
// failing with AZK_ERR_INVALID_INPUT_LAYOUT otherwise or when the address is not
// device memory.
void require_device_range(const void* p, uint64_t off, uint64_t bytes);
// Two byte ranges of device memory overlap (the reference's rangesOverlap on one
// buffer, QM31FRIFold.swift:1280-1294; distinct allocations never overlap).
inline bool ranges_overlap(const void* a, uint64_t aoff, uint64_t abytes, const void* b, uint64_t boff, uint64_t bbytes) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a) + aoff, y = reinterpret_cast<uintptr_t>(b) + boff;
  return x < y + bbytes && y < x + abytes;
}

// Domain tables of size 2^logn, materialised once per context.
const azk_ctx::Domain& domain_tables(azk_ctx* ctx, uint32_t logn);

// Resolved hashing schedule.
struct Sched {
  uint32_t tile_log = 12;
  uint32_t group_log = 12;
  uint32_t threads = 256;
  bool graph = true;
  uint8_t layer_tile[32] = {0};
  uint16_t layer_threads[32] = {0};
  bool persistent_trees = false;
};
// A schedule with no treelet depth and no layer table takes `defaults` (a tuned
// per-layer table from azk_tuned.h) when one is given, and with no thread count
// and no per-layer threads `default_threads` likewise.
Sched resolve_schedule(const azk_schedule* s, const uint8_t* defaults = nullptr, const uint16_t* default_threads = nullptr);
// Threads per CTA of the commit kernel for a layer of 2^logn leaves.
inline uint32_t tree_threads(const Sched& s, uint32_t logn) { return (logn < 32 && s.layer_threads[logn]) ? s.layer_threads[logn] : s.threads; }
// Tile depth used for a tree of 2^logn leaves under a schedule (per-layer table
// first, then the global depth), clamped to [1, logn].
inline uint32_t tree_tile_log(const Sched& s, uint32_t logn) {
  uint32_t t = (logn < 32 && s.layer_tile[logn]) ? s.layer_tile[logn] : s.tile_log;
  if (t > logn) t = logn;
  if (t == 0 && logn > 0) t = 1;
  return t;
}

// FFT work for a set of transforms: one FftJob per (transform, pass); passes of
// all transforms are aligned so every transform's last (low-stage) pass runs at
// the final step.  Inside a step the work items are grouped by pass kernel
// (FftKind: QM31 tiles, small one-limb transforms, one-limb tiles, bulk-copied
// one-limb low passes), each group one contiguous range and one launch.
// Transforms flagged `narrow` (inputs known to be lifted M31 polynomials) take the
// one-limb kernels.
struct FftPlan {
  std::vector<FftJob> jobs;
  std::vector<uint2> work;  // all steps, step-major, kind-major, transform-contiguous
  std::vector<std::array<uint64_t, kFftKinds>> part_off, part_cnt;  // per step and kind
  std::vector<uint8_t> narrow;                                      // per transform
  std::vector<std::vector<std::pair<uint64_t, uint64_t>>> inst_range;  // [step][transform] -> (offset, count)
  std::vector<std::vector<uint8_t>> inst_kind;                         // [step][transform] -> FftKind
  DevBuf d_jobs, d_work;
  DevBuf d_status;  // raised by a pass kernel whose bounded wait ran out
  size_t steps() const { return part_off.size(); }
  void build(const std::vector<FftJob>& transforms, const std::vector<uint8_t>& narrow_flags = {});
  void upload(cudaStream_t s);
  void launch_step(size_t step, cudaStream_t s) const;
  void launch_step_for(size_t step, size_t t, cudaStream_t s) const;
  void launch_all(cudaStream_t s) const {
    for (size_t k = 0; k < steps(); k++) launch_step(k, s);
  }
  // After the stream has finished the passes: fails with AZK_ERR_DEVICE_TIMEOUT (and
  // clears the flag) when a pass kernel gave up waiting for its tile copies.
  // `host_word`: page-locked memory for the readback (else a pageable word).
  void check_status(cudaStream_t s, uint32_t* host_word = nullptr);
};

// Monomial -> interleaved circle FFT-basis coefficients, host-side like the
// reference's CircleCodewordPlan (CircleCodeword.swift:100-127, 187-263).
std::vector<uint32_t> fft_basis_from_monomials(uint32_t logn, const uint32_t* x, uint64_t nx, const uint32_t* y, uint64_t ny);

}  // namespace azk
