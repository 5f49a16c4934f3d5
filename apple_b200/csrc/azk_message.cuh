// Loading fixed-rate messages (<= 136 bytes) into a Keccak state and hashing them
// with SHA3-256 (suffix 0x06) or Keccak-256 (suffix 0x01), as the reference's
// one-block kernels do (HashMerkleKernels.metal:584-909): a message shorter than
// the rate is one permutation; a 136-byte message fills the first block and the
// padding takes a second permutation (absorb_fixed_136, :633-657).
#pragma once
#include "azk_keccak.cuh"

namespace azk {

// XOR `len` message bytes into lanes 0..16.  aligned8: p is 8-byte aligned, so
// whole lanes load as u64; otherwise bytes are gathered one by one.
__device__ __forceinline__ void xor_message(uint64_t (&a)[25], const uint8_t* p, uint32_t len, bool aligned8) {
  uint32_t full = len >> 3;
  if (aligned8) {
    const uint64_t* q = reinterpret_cast<const uint64_t*>(p);
#pragma unroll
    for (uint32_t i = 0; i < 17; i++)
      if (i < full) a[i] ^= __ldg(q + i);
  } else {
#pragma unroll
    for (uint32_t i = 0; i < 17; i++) {
      if (i < full) {
        uint64_t v = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) v |= (uint64_t)__ldg(p + 8 * i + k) << (8 * k);
        a[i] ^= v;
      }
    }
  }
  uint32_t rem = len & 7;
  if (rem) {
    uint64_t v = 0;
    for (uint32_t k = 0; k < rem; k++) v |= (uint64_t)__ldg(p + 8 * full + k) << (8 * k);
    // lane index `full` is dynamic here; select it with an unrolled compare
#pragma unroll
    for (uint32_t i = 0; i < 17; i++)
      if (i == full) a[i] ^= v;
  }
}

// Digest of one message of `len` (<= 136) bytes at p.
__device__ __forceinline__ void hash_message(const uint8_t* p, uint32_t len, uint32_t suffix, bool aligned8, uint64_t (&out)[4]) {
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; i++) a[i] = 0;
  xor_message(a, p, len, aligned8);
  if (len == 136) {
    keccak_f1600(a);
    a[0] ^= suffix;
  } else {
    uint32_t lane = len >> 3;
    uint64_t v = (uint64_t)suffix << (8 * (len & 7));
#pragma unroll
    for (uint32_t i = 0; i < 17; i++)
      if (i == lane) a[i] ^= v;
  }
  a[16] ^= kPadEnd;
  keccak_f1600(a);
#pragma unroll
  for (int i = 0; i < 4; i++) out[i] = a[i];
}

}  // namespace azk
