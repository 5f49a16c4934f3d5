// SHA3 Merkle root of raw leaves for callers that cannot allocate device memory.
//
// Some callers run where cudaMalloc is off limits: inside a host that hands the
// library a fixed memory budget and forbids allocation behind its back, from code
// that must not synchronise the device (cudaMalloc/cudaFree can), or from a
// real-time loop that cannot risk an allocation failure mid-run.  The regular
// Merkle plan allocates its tree, counters and job buffers; this entry point
// instead keeps all of its scratch (the tree's inner nodes and the treelet arrival
// counters) in one fixed array that lives in the library's device image, and takes
// its single job as a kernel argument.  The caller passes the leaves and a 32-byte
// output buffer, both already on the device.
//
// Limits and sharing: at most kNoAllocMaxLeaves leaves (larger requests are
// rejected before anything is launched).  The array is one per device, held by
// every GPU that loads the library until the process exits, and shared by all
// calls on that device: calls whose work overlaps on the GPU (different streams,
// or different host threads on one device) race on it and must be serialised by
// the caller.  Each call clears the counters it needs before its kernel; nodes are
// fully rewritten, so results never depend on an earlier call.
#include <mutex>

#include "azk_runtime.h"

namespace azk {

static constexpr uint64_t kNoAllocMaxLeaves = 1ull << 16;
static constexpr uint32_t kNoAllocTileLog = 9;  // 24 KiB of shared memory: under the default limit
// Arrival counters: with treelets of min(logn, 9) levels a tree of at most 2^16
// leaves has at most 128 treelets, and tree_counter_count() bounds the counters
// (treelets + 64); inner nodes: at most 2^16 - 1 digests.
static constexpr uint64_t kNoAllocCounterBytes = 4ull * ((kNoAllocMaxLeaves >> kNoAllocTileLog) + 64);
static constexpr uint64_t kNoAllocNodeOffset = (kNoAllocCounterBytes + 255) / 256 * 256;
static constexpr uint64_t kNoAllocScratchBytes = kNoAllocNodeOffset + 32ull * kNoAllocMaxLeaves;

// The scratch array: 2 MiB + 768 bytes per device.
static __device__ __align__(256) uint8_t g_merkle_noalloc_scratch[kNoAllocScratchBytes];

// Device addresses of the array, resolved once per device with that device current
// (the array's host-side name is not a device address).  The cached address lives
// as long as the device's context: a cudaDeviceReset in the same process unloads
// the library's device image, so this entry point is not supported after one.
static std::mutex g_noalloc_mu;
static uint8_t* g_noalloc_ptr[64] = {nullptr};

static cudaError_t noalloc_scratch(uint8_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_merkle_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = static_cast<uint8_t*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace azk

extern "C" azk_status azk_merkle_root_noalloc(const void* dev_leaves, uint64_t leaf_count, uint64_t leaf_stride, uint64_t leaf_length,
                                              void* dev_root, void* stream) {
  using namespace azk;
  // failures are reported through azk_last_error_message(NULL)
  auto err = [](azk_status s, const char* m) {
    set_error(nullptr, m);
    return s;
  };
  if (!dev_root || (!dev_leaves && leaf_count * leaf_stride != 0)) return err(AZK_ERR_INVALID_INPUT_LAYOUT, "null device pointer");
  if (leaf_count == 0 || (leaf_count & (leaf_count - 1))) return err(AZK_ERR_INVALID_LEAF_COUNT, "leaf count must be a non-zero power of two");
  if (leaf_count > kNoAllocMaxLeaves)
    return err(AZK_ERR_INVALID_INPUT_LAYOUT, "leaf count exceeds the no-allocation limit of 65536 leaves; use azk_merkle_plan_* instead");
  if (leaf_length > 136) return err(AZK_ERR_UNSUPPORTED_ONE_BLOCK_LENGTH, "fixed-rate SHA3 leaves hold at most 136 bytes");
  if (leaf_stride < leaf_length || leaf_stride > 0xFFFFFFFFull) return err(AZK_ERR_INVALID_INPUT_LAYOUT, "leaf stride must be >= leaf length");

  uint8_t* scratch = nullptr;
  cudaError_t e = noalloc_scratch(&scratch);
  if (e != cudaSuccess) return err(AZK_ERR_COMMAND_EXECUTION_FAILED, cudaGetErrorString(e));
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  uint32_t logn = 0;
  while ((1ull << logn) < leaf_count) logn++;
  uint32_t tl = logn < kNoAllocTileLog ? logn : kNoAllocTileLog;
  if (logn > 0 && tl == 0) tl = 1;
  uint64_t counters = tree_counter_count(logn, tl);
  // the arrival counters must start at zero
  e = cudaMemsetAsync(scratch, 0, 4 * counters, s);
  if (e != cudaSuccess) return err(AZK_ERR_COMMAND_EXECUTION_FAILED, cudaGetErrorString(e));

  TreeJob job{};
  job.logn = logn;
  job.kind = kLeafRaw;
  job.tile_log = tl;
  job.group_log = tl ? tl : 1;
  job.raw = static_cast<const uint8_t*>(dev_leaves);
  job.stride = leaf_stride;
  job.len = (uint32_t)leaf_length;
  job.suffix = 0x06;
  job.aligned8 = (((uintptr_t)dev_leaves & 7) == 0 && (leaf_stride & 7) == 0) ? 1 : 0;
  job.leaf_digests = nullptr;
  job.inner = reinterpret_cast<uint64_t*>(scratch + kNoAllocNodeOffset);
  job.counters = reinterpret_cast<uint32_t*>(scratch);
  job.root_action = kRootNone;
  job.root_out = static_cast<uint64_t*>(dev_root);
  e = launch_tree_direct_raw(job, s);
  if (e != cudaSuccess) {
    set_error(nullptr, std::string("Merkle root kernel launch failed: ") + cudaGetErrorString(e));
    return AZK_ERR_COMMAND_EXECUTION_FAILED;
  }
  return AZK_OK;
}
