// SHA3 Merkle commitment kernels: fused leaf hashing + shared-memory treelets +
// last-arriver upper levels, for raw leaves, prehashed digests, QM31 layers and
// fold-then-hash layers with 16-byte leaves of one QM31 value or 64-byte leaves of
// four (reference: MerkleCommitter.swift:526-1063 and the Metal
// kernels HashMerkleKernels.metal:1064-1292; oracle MerkleOracle.swift:4-141).
//
// Tree layout: level 0 (leaf digests) optional; levels >= 1 in `inner`, level l
// at inner_offset(logn, l), root last.  A digest is 4 little-endian u64 lanes.
//
// Upper levels need no grid-wide wait: each CTA that completes a treelet root
// bumps its group's arrival counter; the CTA that arrives last reads the group's
// roots (written by the others before their fence + atomic) and reduces them.
// Counters reset themselves, so the same job list can be relaunched (and
// captured in a CUDA graph).
#include "azk_field.cuh"
#include "azk_internal.h"
#include "azk_message.cuh"

namespace azk {

struct Dig {
  uint64_t w[4];
};

__device__ __forceinline__ void st_dig(uint64_t* p, const uint64_t (&d)[4]) {
  reinterpret_cast<ulonglong2*>(p)[0] = make_ulonglong2(d[0], d[1]);
  reinterpret_cast<ulonglong2*>(p)[1] = make_ulonglong2(d[2], d[3]);
}
__device__ __forceinline__ void ld_dig(const uint64_t* p, uint64_t (&d)[4]) {
  ulonglong2 a = reinterpret_cast<const ulonglong2*>(p)[0], b = reinterpret_cast<const ulonglong2*>(p)[1];
  d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y;
}
// L2 read of a digest written by another CTA in this launch.
__device__ __forceinline__ void ld_dig_cg(const uint64_t* p, uint64_t (&d)[4]) {
  ulonglong2 a = __ldcg(reinterpret_cast<const ulonglong2*>(p));
  ulonglong2 b = __ldcg(reinterpret_cast<const ulonglong2*>(p) + 1);
  d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y;
}

template <uint32_t KIND>
__device__ __forceinline__ void leaf_digest(const TreeJob& job, uint64_t leaf, const uint32_t (&ch)[4], uint64_t (&d)[4]) {
  if constexpr (KIND == kLeafQM31) {
    uint4 v = __ldg(job.layer + leaf);
    sha3_16((uint64_t)v.x | ((uint64_t)v.y << 32), (uint64_t)v.z | ((uint64_t)v.w << 32), d);
  } else if constexpr (KIND == kLeafFold) {
    uint4 p = __ldg(job.layer + 2 * leaf), q = __ldg(job.layer + 2 * leaf + 1);
    uint32_t t = __ldg(job.inv + leaf);
    qm31 r = fri_fold_pair(qm31{p.x, p.y, p.z, p.w}, qm31{q.x, q.y, q.z, q.w}, t, qm31{ch[0], ch[1], ch[2], ch[3]});
    job.out_layer[leaf] = make_uint4(r.a, r.b, r.c, r.d);
    sha3_16((uint64_t)r.a | ((uint64_t)r.b << 32), (uint64_t)r.c | ((uint64_t)r.d << 32), d);
  } else if constexpr (KIND == kLeafDigest) {
    ld_dig(reinterpret_cast<const uint64_t*>(job.raw) + 4 * leaf, d);
  } else {
    hash_message(job.raw + leaf * job.stride, job.len, job.suffix, job.aligned8 != 0, d);
  }
}

// Reduce `count` digests in buffer a (scratch b holds count/2) level by level,
// storing each level into the job's inner nodes.  Returns the buffer holding the
// single remaining digest.  `level`/`idx0`: level and first node index of the
// input digests.
__device__ __noinline__ uint64_t* reduce_levels(uint64_t* a, uint64_t* b, uint32_t count, const TreeJob& job, uint32_t level, uint64_t idx0) {
  uint64_t* src = a;
  uint64_t* dst = b;
  while (count > 1) {
    count >>= 1;
    idx0 >>= 1;
    level++;
    uint64_t* lv = job.inner + 4 * (inner_offset(job.logn, level) + idx0);
    for (uint32_t i = threadIdx.x; i < count; i += blockDim.x) {
      uint64_t l[4], r[4], d[4];
      ld_dig(src + 8 * i, l);
      ld_dig(src + 8 * i + 4, r);
      sha3_pair(l, r, d);
      st_dig(dst + 4 * i, d);
      st_dig(lv + 4 * i, d);
    }
    __syncthreads();
    uint64_t* t = src;
    src = dst;
    dst = t;
  }
  return src;
}

__device__ __noinline__ void root_action(const TreeJob& job, const uint64_t* rootp) {
  uint64_t root[4];
  ld_dig(rootp, root);
  if (job.root_out) st_dig(job.root_out, root);
  if (job.root_action == kRootNone) return;
  Transcript t = *job.transcript;
  uint32_t ch[4];
  if (job.root_action == kRootCircleRound)
    circle_round(t, job.round, root, ch);
  else
    qm31_round(t, job.round, job.frame_in_count, root, ch);
  *job.transcript = t;
  for (int k = 0; k < 4; k++) job.challenge_out[k] = ch[k];
}

// Sets up the sponge input of one leaf (message lanes, suffix and end padding)
// and returns how many permutations it takes (2 for a 136-byte raw leaf).
template <uint32_t KIND>
__device__ __forceinline__ uint32_t leaf_setup(const TreeJob& job, uint64_t leaf, const uint32_t (&ch)[4], uint64_t (&a)[25]) {
  if constexpr (KIND == kLeafQM31 || KIND == kLeafFold) {
    uint4 v;
    if constexpr (KIND == kLeafQM31) {
      v = __ldg(job.layer + leaf);
    } else {
      uint4 p = __ldg(job.layer + 2 * leaf), q = __ldg(job.layer + 2 * leaf + 1);
      qm31 r = fri_fold_pair(qm31{p.x, p.y, p.z, p.w}, qm31{q.x, q.y, q.z, q.w}, __ldg(job.inv + leaf), qm31{ch[0], ch[1], ch[2], ch[3]});
      v = make_uint4(r.a, r.b, r.c, r.d);
      job.out_layer[leaf] = v;
    }
    a[0] = (uint64_t)v.x | ((uint64_t)v.y << 32);
    a[1] = (uint64_t)v.z | ((uint64_t)v.w << 32);
    a[2] = 0x06;
    a[16] = kPadEnd;
    return 1;
  } else if constexpr (KIND == kLeafQM31x4 || KIND == kLeafFoldx4) {
    // leaf = values 4*leaf .. 4*leaf+3 (64 bytes, 8 lanes)
#pragma unroll
    for (uint32_t m = 0; m < 4; m++) {
      const uint64_t e = 4 * leaf + m;
      uint4 v;
      if constexpr (KIND == kLeafQM31x4) {
        v = __ldg(job.layer + e);
      } else {
        uint4 p = __ldg(job.layer + 2 * e), q = __ldg(job.layer + 2 * e + 1);
        qm31 r = fri_fold_pair(qm31{p.x, p.y, p.z, p.w}, qm31{q.x, q.y, q.z, q.w}, __ldg(job.inv + e), qm31{ch[0], ch[1], ch[2], ch[3]});
        v = make_uint4(r.a, r.b, r.c, r.d);
        job.out_layer[e] = v;
      }
      a[2 * m] = (uint64_t)v.x | ((uint64_t)v.y << 32);
      a[2 * m + 1] = (uint64_t)v.z | ((uint64_t)v.w << 32);
    }
    a[8] = 0x06;
    a[16] = kPadEnd;
    return 1;
  } else {
    xor_message(a, job.raw + leaf * job.stride, job.len, job.aligned8 != 0);
    if (job.len == 136) return 2;
    const uint32_t lane = job.len >> 3;
    const uint64_t v = (uint64_t)job.suffix << (8 * (job.len & 7));
#pragma unroll
    for (uint32_t i = 0; i < 17; i++)
      if (i == lane) a[i] ^= v;
    a[16] ^= kPadEnd;
    return 1;
  }
}

// Subtrees of height h = min(2, log2(items)), one per thread.  Items are the
// tile's leaves, or (from_nodes) digests already in the tree at level `base`.  The
// subtree's inner nodes are stored (levels base+1 .. base+h, first node idx0 >> l)
// and its root written to `out` in shared memory.  A 4-item subtree runs as a
// 7-step loop around ONE permutation site (leaf, leaf, pair, leaf, leaf, pair,
// pair), which keeps the kernel's code small enough for the instruction cache.
template <uint32_t KIND, int THREADS>
__device__ __noinline__ uint32_t subtree_phase(const TreeJob& job, uint32_t items, uint32_t base, uint64_t idx0, const uint64_t* nodes, bool from_nodes,
                                               uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t* out) {
  const uint32_t ch[4] = {c0, c1, c2, c3};
  const uint32_t h = items >= 4 ? 2u : (items >= 2 ? 1u : 0u);
  const uint32_t groups = items >> h;
  const bool item_is_digest = from_nodes || KIND == kLeafDigest;
  const uint64_t* digests = from_nodes ? nodes : reinterpret_cast<const uint64_t*>(job.raw) + 4 * idx0;
  uint64_t* l1 = job.inner + 4 * (inner_offset(job.logn, base + 1) + (idx0 >> 1));
  uint64_t* l2 = job.inner + 4 * (inner_offset(job.logn, base + 2) + (idx0 >> 2));
  // step k: item index within the subtree (leaf steps) and the step's kind
  //   k:     0  1  2  3  4  5  6        (h == 2)
  //   item:  0  1  -  2  3  -  -
  const uint32_t steps = h == 2 ? 7 : (h == 1 ? 3 : 1);
  for (uint32_t j = threadIdx.x; j < groups; j += THREADS) {
    uint64_t X[4] = {0, 0, 0, 0}, Y[4] = {0, 0, 0, 0}, P[4] = {0, 0, 0, 0};
#pragma unroll 1
    for (uint32_t k = 0; k < steps; k++) {
      const bool pair = (h == 2) ? (k == 2 || k == 5 || k == 6) : (h == 1 && k == 2);
      const uint32_t item = k < 2 ? k : k - 1;  // leaf steps only (h == 2: k = 0, 1, 3, 4)
      const uint64_t leaf = idx0 + (uint64_t)j * (1u << h) + item;
      uint64_t d[4];
      if (!pair && item_is_digest) {
        ld_dig_cg(digests + 4 * ((uint64_t)j * (1u << h) + item), d);
      } else {
        uint64_t a[25];
#pragma unroll
        for (int i = 0; i < 25; i++) a[i] = 0;
        uint32_t perms = 1;
        if (pair) {
          const bool top = (h == 2 && k == 6);
#pragma unroll
          for (int i = 0; i < 4; i++) {
            a[i] = top ? P[i] : X[i];
            a[4 + i] = Y[i];
          }
          a[8] = 0x06;
          a[16] = kPadEnd;
        } else {
          perms = leaf_setup<KIND>(job, leaf, ch, a);
        }
#pragma unroll 1
        for (uint32_t b = 0; b < perms; b++) {
          if (b == 1) {
            a[0] ^= job.suffix;
            a[16] ^= kPadEnd;
          }
          keccak_f1600(a);
        }
#pragma unroll
        for (int i = 0; i < 4; i++) d[i] = a[i];
        if (!pair && job.leaf_digests) st_dig(job.leaf_digests + 4 * leaf, d);
      }
      // route the step's digest
      const bool toX = (h == 2) ? (k == 0 || k == 3) : (h == 1 && k == 0);
      const bool toY = (h == 2) ? (k == 1 || k == 4 || k == 5) : (h == 1 && k == 1);
      const bool toP = (h == 2 && k == 2);
#pragma unroll
      for (int i = 0; i < 4; i++) {
        X[i] = toX ? d[i] : X[i];
        Y[i] = toY ? d[i] : Y[i];
        P[i] = toP ? d[i] : P[i];
      }
      if (h == 2 && k == 2) st_dig(l1 + 8 * j, d);
      if (h == 2 && k == 5) st_dig(l1 + 8 * j + 4, d);
      if (h == 2 && k == 6) st_dig(l2 + 4 * j, d);
      if (h == 1 && k == 2) st_dig(l1 + 4 * j, d);
      if (k + 1 == steps) st_dig(out + 4 * j, d);
    }
  }
  __syncthreads();
  return h;
}

// One tile of one job: leaf digests, treelet, then the last-arriver climb.
// Shared memory: 2^(tl-2) digests + half as many for the ping-pong (12 bytes per leaf).
template <uint32_t KIND, int THREADS>
__device__ __forceinline__ void tree_tile_body(const TreeJob& job, const uint64_t tile) {
  extern __shared__ __align__(16) uint64_t sm[];
  __shared__ uint32_t s_last;
  __shared__ uint32_t s_ch[4];
  const uint32_t tl = job.tile_log < job.logn ? job.tile_log : job.logn;
  const uint32_t T = 1u << tl;
  const uint32_t Q = T >= 4 ? T / 4 : 1;
  uint64_t* bufA = sm;           // Q digests
  uint64_t* bufB = sm + 4 * Q;   // Q/2 digests

  uint32_t ch[4] = {0, 0, 0, 0};
  if constexpr (KIND == kLeafFold || KIND == kLeafFoldx4) {
    if (threadIdx.x < 4) s_ch[threadIdx.x] = __ldcg(job.fold_ch + threadIdx.x);
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; k++) ch[k] = s_ch[k];
  }

  // 1) leaf digests and the two lowest levels of this tile, per thread
  const uint64_t first = tile * T;
  uint32_t h = subtree_phase<KIND, THREADS>(job, T, 0, first, nullptr, false, ch[0], ch[1], ch[2], ch[3], bufA);
  // 2) treelet
  uint64_t* res = reduce_levels(bufA, bufB, T >> h, job, h, first >> h);
  // 3) climb: last arriver of each group continues
  uint32_t level = tl;
  uint64_t idx = tile;
  uint64_t cnt_off = 0;
  while (level < job.logn) {
    uint32_t glog = job.group_log;
    if (glog > job.logn - level) glog = job.logn - level;
    if (glog > tl) glog = tl;  // the group must fit the shared buffers (host keeps tl >= 1)
    const uint32_t G = 1u << glog;
    const uint64_t gidx = idx >> glog;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      uint32_t old = atomicAdd(job.counters + cnt_off + gidx, 1u);
      s_last = (old == G - 1) ? 1u : 0u;
      if (s_last) job.counters[cnt_off + gidx] = 0;  // reset for the next launch
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const uint64_t* lv = job.inner + 4 * (inner_offset(job.logn, level) + gidx * G);
    uint32_t hg = subtree_phase<KIND, THREADS>(job, G, level, gidx * G, lv, true, 0, 0, 0, 0, bufA);
    res = reduce_levels(bufA, bufB, G >> hg, job, level + hg, (gidx * G) >> hg);
    cnt_off += (1ull << (job.logn - level)) >> glog;
    level += glog;
    idx = gidx;
  }
  if (threadIdx.x == 0) root_action(job, res);
}

template <uint32_t KIND, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) tree_tiles_kernel(const TreeJob* __restrict__ jobs, const uint2* __restrict__ work) {
  const uint2 w = work[blockIdx.x];
  tree_tile_body<KIND, THREADS>(jobs[w.x], w.y);
}

// Persistent form: a grid of the resident CTAs pulls work items from a device
// counter (queue[0]) until the list is done.  Nothing waits on anything: the
// last-arriver climb is unchanged, and the last CTA to leave (queue[1] counts
// them) resets both counters, so a captured launch sequence replays.
template <uint32_t KIND, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) tree_queue_kernel(const TreeJob* __restrict__ jobs, const uint2* __restrict__ work,
                                                                            uint32_t nwork, uint32_t* __restrict__ queue) {
  __shared__ uint32_t s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t item = s_item;
    __syncthreads();  // every thread has the item (and the last one's shared memory is free)
    if (item >= nwork) break;
    const uint2 w = work[item];
    tree_tile_body<KIND, THREADS>(jobs[w.x], w.y);
  }
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(queue + 1, 1u) == gridDim.x - 1) {
      queue[0] = 0;
      queue[1] = 0;
    }
  }
}

// Single job passed by value, tile = blockIdx.x: needs no job or work-list buffer.
template <uint32_t KIND, int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) tree_direct_kernel(const TreeJob job) {
  tree_tile_body<KIND, THREADS>(job, blockIdx.x);
}

static constexpr int kMaxTreeLog = 13;
static constexpr int kMaxTreeSmem = 12 << kMaxTreeLog;  // 2^11 digests + 2^10 digests

template <uint32_t KIND>
static cudaError_t prepare_kind() {
  cudaError_t e = cudaSuccess;
  for (auto k : {tree_tiles_kernel<KIND, 128>, tree_tiles_kernel<KIND, 256>, tree_tiles_kernel<KIND, 512>}) {
    cudaError_t r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxTreeSmem);
    if (r != cudaSuccess) e = r;
  }
  for (auto k : {tree_queue_kernel<KIND, 128>, tree_queue_kernel<KIND, 256>, tree_queue_kernel<KIND, 512>}) {
    cudaError_t r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxTreeSmem);
    if (r != cudaSuccess) e = r;
  }
  return e;
}

// Opt the tree kernels into > 48 KiB of dynamic shared memory once, outside any
// stream capture.
cudaError_t prepare_tree_kernels() {
  cudaError_t e = prepare_kind<kLeafRaw>();
  if (e == cudaSuccess) e = prepare_kind<kLeafQM31>();
  if (e == cudaSuccess) e = prepare_kind<kLeafFold>();
  if (e == cudaSuccess) e = prepare_kind<kLeafDigest>();
  if (e == cudaSuccess) e = prepare_kind<kLeafQM31x4>();
  if (e == cudaSuccess) e = prepare_kind<kLeafFoldx4>();
  return e;
}

// Resident CTAs of a persistent launch: the occupancy of the kernel at this
// shared-memory size times the SMs, no more than the work items.
template <class K>
static uint32_t resident_grid(K kernel, int threads, size_t smem, uint32_t nwork) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
    if (sms < 1) sms = 148;
  }
  const uint64_t g = (uint64_t)sms * (uint64_t)per_sm;
  return (uint32_t)(g < nwork ? g : nwork);
}

template <uint32_t KIND>
static cudaError_t launch_kind(const TreeJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t max_tile_log, uint32_t threads, uint32_t* queue,
                               cudaStream_t s) {
  size_t smem = max_tile_log >= 2 ? ((size_t)12 << max_tile_log) : 48;  // T/4 digests + T/8 digests
  if (queue) {
    if (threads == 128)
      tree_queue_kernel<KIND, 128><<<resident_grid(tree_queue_kernel<KIND, 128>, 128, smem, nwork), 128, smem, s>>>(d_jobs, d_work, nwork, queue);
    else if (threads == 512)
      tree_queue_kernel<KIND, 512><<<resident_grid(tree_queue_kernel<KIND, 512>, 512, smem, nwork), 512, smem, s>>>(d_jobs, d_work, nwork, queue);
    else
      tree_queue_kernel<KIND, 256><<<resident_grid(tree_queue_kernel<KIND, 256>, 256, smem, nwork), 256, smem, s>>>(d_jobs, d_work, nwork, queue);
    return cudaGetLastError();
  }
  if (threads == 128)
    tree_tiles_kernel<KIND, 128><<<nwork, 128, smem, s>>>(d_jobs, d_work);
  else if (threads == 512)
    tree_tiles_kernel<KIND, 512><<<nwork, 512, smem, s>>>(d_jobs, d_work);
  else
    tree_tiles_kernel<KIND, 256><<<nwork, 256, smem, s>>>(d_jobs, d_work);
  return cudaGetLastError();
}

cudaError_t launch_tree_jobs(const TreeJob* d_jobs, const uint2* d_work, uint32_t nwork, uint32_t max_tile_log, uint32_t kind, uint32_t threads,
                             cudaStream_t s, uint32_t* d_queue) {
  if (nwork == 0) return cudaSuccess;
  if (max_tile_log > kMaxTreeLog) return cudaErrorInvalidValue;
  switch (kind) {
    case kLeafRaw: return launch_kind<kLeafRaw>(d_jobs, d_work, nwork, max_tile_log, threads, d_queue, s);
    case kLeafQM31: return launch_kind<kLeafQM31>(d_jobs, d_work, nwork, max_tile_log, threads, d_queue, s);
    case kLeafFold: return launch_kind<kLeafFold>(d_jobs, d_work, nwork, max_tile_log, threads, d_queue, s);
    case kLeafDigest: return launch_kind<kLeafDigest>(d_jobs, d_work, nwork, max_tile_log, threads, d_queue, s);
    case kLeafQM31x4: return launch_kind<kLeafQM31x4>(d_jobs, d_work, nwork, max_tile_log, threads, d_queue, s);
    case kLeafFoldx4: return launch_kind<kLeafFoldx4>(d_jobs, d_work, nwork, max_tile_log, threads, d_queue, s);
    default: return cudaErrorInvalidValue;
  }
}

// One raw-leaf tree, job by value, 256 threads, treelets of at most 2^9 leaves
// (24 KiB of dynamic shared memory: under the default limit, no opt-in needed).
cudaError_t launch_tree_direct_raw(const TreeJob& job, cudaStream_t s) {
  if (job.tile_log > 9 || (job.logn > 0 && job.tile_log == 0)) return cudaErrorInvalidValue;
  uint32_t tl = job.tile_log < job.logn ? job.tile_log : job.logn;
  unsigned tiles = 1u << (job.logn - tl);
  tree_direct_kernel<kLeafRaw, 256><<<tiles, 256, tl >= 2 ? ((size_t)12 << tl) : 48, s>>>(job);
  return cudaGetLastError();
}

// Sibling paths for leaves of a committed tree: out[k][level] = digest of the
// sibling at `level` (bottom-up), depth = job.logn digests per index.  Level 0
// comes from stored leaf digests, or is recomputed from the leaf source.
__global__ void gather_openings_kernel(const TreeJob* __restrict__ jobp, const uint64_t* __restrict__ idx, uint32_t nidx, uint64_t* __restrict__ out) {
  const TreeJob& job = *jobp;
  uint32_t depth = job.logn;
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (uint64_t)nidx * depth) return;
  uint32_t k = (uint32_t)(t / depth), level = (uint32_t)(t % depth);
  uint64_t leaf = idx[k];
  uint64_t node = (leaf >> level) ^ 1ull;
  uint64_t d[4];
  if (level == 0) {
    if (job.leaf_digests) {
      ld_dig(job.leaf_digests + 4 * node, d);
    } else {
      uint32_t ch[4] = {0, 0, 0, 0};
      if (job.kind == kLeafQM31)
        leaf_digest<kLeafQM31>(job, node, ch, d);
      else if (job.kind == kLeafDigest)
        leaf_digest<kLeafDigest>(job, node, ch, d);
      else
        leaf_digest<kLeafRaw>(job, node, ch, d);
    }
  } else {
    ld_dig(job.inner + 4 * (inner_offset(job.logn, level) + node), d);
  }
  st_dig(out + 4 * ((uint64_t)k * depth + level), d);
}

cudaError_t launch_gather_openings(const TreeJob* d_job, const uint64_t* d_idx, uint32_t nidx, uint64_t* d_out, cudaStream_t s) {
  // depth is read on the device; launch enough threads for the deepest tree (31 levels)
  uint64_t total = (uint64_t)nidx * 32;
  if (total == 0) return cudaSuccess;
  gather_openings_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(d_job, d_idx, nidx, d_out);
  return cudaGetLastError();
}

}  // namespace azk
