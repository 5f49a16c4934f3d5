// Batch Keccak-f[1600] permutations and fixed-rate SHA3-256 / Keccak-256 batch
// hashing (KeccakF1600PermutationBatcher.swift:73-294, SHA3BatchHasher.swift:81-264;
// Metal kernels HashMerkleKernels.metal:428-478, 758-909).
//
// One permutation per thread, state in registers.  Contiguous 200-byte states are
// staged through shared memory with 16-byte coalesced loads; other strides load
// lane by lane.
#include "azk_internal.h"
#include "azk_message.cuh"

namespace azk {

// Contiguous states (stride 200, 16-byte aligned base): the CTA copies its
// blockDim.x states to shared memory with uint4 loads, each thread permutes one.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) keccak_permute_staged(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, uint64_t count) {
  extern __shared__ uint4 smem4[];
  uint64_t first = (uint64_t)blockIdx.x * THREADS;
  uint32_t n = (uint32_t)((count - first) < (uint64_t)THREADS ? (count - first) : (uint64_t)THREADS);
  const uint4* src = reinterpret_cast<const uint4*>(in + first * 200);
  uint32_t vecs = n * 200 / 16;  // n * 12.5: states pair up into whole vectors
  uint32_t tail_bytes = (n * 200) % 16;
  for (uint32_t v = threadIdx.x; v < vecs; v += THREADS) smem4[v] = __ldg(src + v);
  if (tail_bytes && threadIdx.x == 0) {
    const uint64_t* s8 = reinterpret_cast<const uint64_t*>(in + first * 200 + (uint64_t)vecs * 16);
    reinterpret_cast<uint64_t*>(smem4 + vecs)[0] = s8[0];
  }
  __syncthreads();
  if (threadIdx.x < n) {
    uint64_t* st = reinterpret_cast<uint64_t*>(smem4) + threadIdx.x * 25;
    uint64_t a[25];
#pragma unroll
    for (int i = 0; i < 25; i++) a[i] = st[i];
    keccak_f1600(a);
#pragma unroll
    for (int i = 0; i < 25; i++) st[i] = a[i];
  }
  __syncthreads();
  uint4* dst = reinterpret_cast<uint4*>(out + first * 200);
  for (uint32_t v = threadIdx.x; v < vecs; v += THREADS) dst[v] = smem4[v];
  if (tail_bytes && threadIdx.x == 0) {
    uint64_t* d8 = reinterpret_cast<uint64_t*>(out + first * 200 + (uint64_t)vecs * 16);
    d8[0] = reinterpret_cast<uint64_t*>(smem4 + vecs)[0];
  }
}

// Any stride that is a multiple of 8 bytes: lane-by-lane loads and stores; bytes
// of an output stride beyond 200 are zeroed (the reference zeroes its output
// buffer when outputStride > 200, KeccakF1600PermutationBatcher.swift:161-164).
__global__ void __launch_bounds__(256) keccak_permute_strided(const uint8_t* __restrict__ in, uint64_t in_stride, uint8_t* __restrict__ out,
                                                              uint64_t out_stride, uint64_t count) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t* s = reinterpret_cast<const uint64_t*>(in + i * in_stride);
  uint64_t a[25];
#pragma unroll
  for (int k = 0; k < 25; k++) a[k] = __ldg(s + k);
  keccak_f1600(a);
  uint64_t* d = reinterpret_cast<uint64_t*>(out + i * out_stride);
#pragma unroll
  for (int k = 0; k < 25; k++) d[k] = a[k];
  for (uint64_t k = 25; k < out_stride / 8; k++) d[k] = 0;
}

cudaError_t launch_keccak_permute(const uint8_t* in, uint64_t in_stride, uint8_t* out, uint64_t out_stride, uint64_t count, uint32_t threads,
                                  cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  bool staged = in_stride == 200 && out_stride == 200 && ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0);
  if (staged) {
    constexpr int T = 128;
    uint64_t blocks = (count + T - 1) / T;
    keccak_permute_staged<T><<<(unsigned)blocks, T, T * 200, s>>>(in, out, count);
  } else {
    uint32_t t = threads ? threads : 256;
    if (t > 256) t = 256;
    keccak_permute_strided<<<(unsigned)((count + t - 1) / t), t, 0, s>>>(in, in_stride, out, out_stride, count);
  }
  return cudaGetLastError();
}

// One message per thread; digest plus zeroed padding up to out_stride.
template <int LEN>
__global__ void __launch_bounds__(256) hash_batch_fixed(const uint8_t* __restrict__ in, uint64_t stride, uint32_t suffix, uint8_t* __restrict__ out,
                                                        uint64_t out_stride, uint64_t count, int aligned8) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint64_t d[4];
  hash_message(in + i * stride, LEN, suffix, aligned8 != 0, d);
  uint8_t* o = out + i * out_stride;
  if ((out_stride & 7) == 0 && ((uintptr_t)out & 7) == 0) {
    uint64_t* o8 = reinterpret_cast<uint64_t*>(o);
#pragma unroll
    for (int k = 0; k < 4; k++) o8[k] = d[k];
    for (uint64_t k = 4; k < out_stride / 8; k++) o8[k] = 0;
  } else {
    for (int k = 0; k < 32; k++) o[k] = (uint8_t)(d[k >> 3] >> (8 * (k & 7)));
    for (uint64_t k = 32; k < out_stride; k++) o[k] = 0;
  }
}

__global__ void __launch_bounds__(256) hash_batch_any(const uint8_t* __restrict__ in, uint64_t stride, uint32_t len, uint32_t suffix,
                                                      uint8_t* __restrict__ out, uint64_t out_stride, uint64_t count, int aligned8) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint64_t d[4];
  hash_message(in + i * stride, len, suffix, aligned8 != 0, d);
  uint8_t* o = out + i * out_stride;
  for (int k = 0; k < 32; k++) o[k] = (uint8_t)(d[k >> 3] >> (8 * (k & 7)));
  for (uint64_t k = 32; k < out_stride; k++) o[k] = 0;
}

cudaError_t launch_hash_batch(const uint8_t* in, uint64_t stride, uint32_t len, uint32_t suffix, uint8_t* out, uint64_t out_stride, uint64_t count,
                              uint32_t threads, cudaStream_t s) {
  if (count == 0) return cudaSuccess;
  uint32_t t = threads ? threads : 256;
  if (t > 256) t = 256;
  unsigned blocks = (unsigned)((count + t - 1) / t);
  int aligned8 = (((uintptr_t)in & 7) == 0 && (stride & 7) == 0) ? 1 : 0;
  switch (len) {
    case 32: hash_batch_fixed<32><<<blocks, t, 0, s>>>(in, stride, suffix, out, out_stride, count, aligned8); break;
    case 64: hash_batch_fixed<64><<<blocks, t, 0, s>>>(in, stride, suffix, out, out_stride, count, aligned8); break;
    case 128: hash_batch_fixed<128><<<blocks, t, 0, s>>>(in, stride, suffix, out, out_stride, count, aligned8); break;
    case 136: hash_batch_fixed<136><<<blocks, t, 0, s>>>(in, stride, suffix, out, out_stride, count, aligned8); break;
    default: hash_batch_any<<<blocks, t, 0, s>>>(in, stride, len, suffix, out, out_stride, count, aligned8); break;
  }
  return cudaGetLastError();
}

}  // namespace azk
