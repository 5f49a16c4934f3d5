// Keccak-f[1600] and the SHA3-256 / Keccak-256 fixed-rate helpers for sm_100a.
//
// The state lives in 25 u64 registers per thread (one permutation per thread).
// Each 64-bit lane is two 32-bit halves: XORs map to LOP3 (three-input XOR, and
// the chi term a ^ (~b & c) is one LOP3 per half) and the rotations to funnel
// shifts, which is the integer-issue mix the roofline counts (180 32-bit ops per
// round, 4,320 per permutation).
//
// Semantics follow the reference's CPU oracle (SHA3Oracle.swift:242-280) and its
// Metal kernels (HashMerkleKernels.metal:308-348): theta, rho+pi, chi, iota with
// the standard round constants.  Functions are __host__ __device__ so the same
// code is unit-tested on the CPU.
#pragma once
#include <stdint.h>

#ifndef __CUDACC__
#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __forceinline__
#define __forceinline__ inline __attribute__((always_inline))
#endif
#endif

namespace azk {

#if defined(__CUDACC__)
__constant__ static const uint64_t kKeccakRC[24] = {
#else
static const uint64_t kKeccakRC[24] = {
#endif
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808AULL, 0x8000000080008000ULL,
    0x000000000000808BULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008AULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000AULL,
    0x000000008000808BULL, 0x800000000000008BULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800AULL, 0x800000008000000AULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};

// Rotate left by a compile-time amount, as two funnel shifts on the 32-bit halves.
template <int N>
__host__ __device__ __forceinline__ uint64_t rotl(uint64_t v) {
  constexpr int n = N & 63;
  if constexpr (n == 0) {
    return v;
  } else {
#if defined(__CUDA_ARCH__)
  uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
  if (n >= 32) { uint32_t t = lo; lo = hi; hi = t; }
  constexpr int m = n & 31;
  if constexpr (m == 0) {
    return ((uint64_t)hi << 32) | lo;
  } else {
    uint32_t nhi = __funnelshift_l(lo, hi, m);
    uint32_t nlo = __funnelshift_l(hi, lo, m);
    return ((uint64_t)nhi << 32) | nlo;
  }
#else
  return (v << n) | (v >> (64 - n));
#endif
  }
}

// rho offset of lane x + 5y
#define AZK_RHO(i)                                                                                       \
  ((i) == 0 ? 0 : (i) == 1 ? 1 : (i) == 2 ? 62 : (i) == 3 ? 28 : (i) == 4 ? 27 : (i) == 5 ? 36 :        \
   (i) == 6 ? 44 : (i) == 7 ? 6 : (i) == 8 ? 55 : (i) == 9 ? 20 : (i) == 10 ? 3 : (i) == 11 ? 10 :     \
   (i) == 12 ? 43 : (i) == 13 ? 25 : (i) == 14 ? 39 : (i) == 15 ? 41 : (i) == 16 ? 45 : (i) == 17 ? 15 : \
   (i) == 18 ? 21 : (i) == 19 ? 8 : (i) == 20 ? 18 : (i) == 21 ? 2 : (i) == 22 ? 61 : (i) == 23 ? 56 : 14)

// pi: lane (x, y) moves to (y, 2x + 3y mod 5)
#define AZK_PI_DST(x, y) ((y) + 5 * ((2 * (x) + 3 * (y)) % 5))

template <int I>
struct RhoPi {
  static constexpr int x = I % 5, y = I / 5;
  static constexpr int dst = AZK_PI_DST(x, y);
  static constexpr int rho = AZK_RHO(I);
};

template <int I>
__host__ __device__ __forceinline__ void rho_pi_lane(const uint64_t (&a)[25], const uint64_t (&d)[5], uint64_t (&b)[25]) {
  b[RhoPi<I>::dst] = rotl<RhoPi<I>::rho>(a[I] ^ d[I % 5]);
}

template <int... Is>
struct LaneSeq {};

template <int... Is>
__host__ __device__ __forceinline__ void rho_pi_all(const uint64_t (&a)[25], const uint64_t (&d)[5], uint64_t (&b)[25], LaneSeq<Is...>) {
  (rho_pi_lane<Is>(a, d, b), ...);
}

// Three-input logic on the 32-bit halves as single LOP3 instructions (truth
// tables over inputs a = 0xF0, b = 0xCC, c = 0xAA): 0x96 = a ^ b ^ c,
// 0xD2 = a ^ (~b & c).  Written out so that theta's column terms are folded into
// each lane's XOR (one LOP3 per half) instead of being combined first and XORed
// in afterwards (two), which is the 180-operation round the roofline counts.
__device__ __forceinline__ uint32_t lop3_xor3(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t lop3_chi(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm("lop3.b32 %0, %1, %2, %3, 0xD2;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint64_t xor3_64(uint64_t a, uint64_t b, uint64_t c) {
  return ((uint64_t)lop3_xor3((uint32_t)(a >> 32), (uint32_t)(b >> 32), (uint32_t)(c >> 32)) << 32) |
         lop3_xor3((uint32_t)a, (uint32_t)b, (uint32_t)c);
}
__device__ __forceinline__ uint64_t chi_64(uint64_t a, uint64_t b, uint64_t c) {
  return ((uint64_t)lop3_chi((uint32_t)(a >> 32), (uint32_t)(b >> 32), (uint32_t)(c >> 32)) << 32) |
         lop3_chi((uint32_t)a, (uint32_t)b, (uint32_t)c);
}

// rho-pi of lane I after theta: a[I] ^ C[x-1] ^ rotl1(C[x+1]) in one three-input XOR
template <int I>
__device__ __forceinline__ void rho_pi_lane3(const uint64_t (&a)[25], const uint64_t (&c)[5], const uint64_t (&r1)[5], uint64_t (&b)[25]) {
  constexpr int x = I % 5;
  b[RhoPi<I>::dst] = rotl<RhoPi<I>::rho>(xor3_64(a[I], c[(x + 4) % 5], r1[(x + 1) % 5]));
}
template <int... Is>
__device__ __forceinline__ void rho_pi_all3(const uint64_t (&a)[25], const uint64_t (&c)[5], const uint64_t (&r1)[5], uint64_t (&b)[25], LaneSeq<Is...>) {
  (rho_pi_lane3<Is>(a, c, r1, b), ...);
}

__host__ __device__ __forceinline__ void keccak_round(uint64_t (&a)[25], uint64_t rc) {
#if defined(__CUDA_ARCH__)
  uint64_t c[5], r1[5], b[25];
#pragma unroll
  for (int x = 0; x < 5; x++) c[x] = xor3_64(xor3_64(a[x], a[x + 5], a[x + 10]), a[x + 15], a[x + 20]);
#pragma unroll
  for (int x = 0; x < 5; x++) r1[x] = rotl<1>(c[x]);
  rho_pi_all3(a, c, r1, b, LaneSeq<0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24>{});
#pragma unroll
  for (int y = 0; y < 25; y += 5) {
#pragma unroll
    for (int x = 0; x < 5; x++) a[y + x] = chi_64(b[y + x], b[y + (x + 1) % 5], b[y + (x + 2) % 5]);
  }
  a[0] ^= rc;
#else
  uint64_t c[5], d[5], b[25];
#pragma unroll
  for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
  for (int x = 0; x < 5; x++) d[x] = c[(x + 4) % 5] ^ rotl<1>(c[(x + 1) % 5]);
  rho_pi_all(a, d, b, LaneSeq<0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24>{});
#pragma unroll
  for (int y = 0; y < 25; y += 5) {
#pragma unroll
    for (int x = 0; x < 5; x++) a[y + x] = b[y + x] ^ (~b[y + (x + 1) % 5] & b[y + (x + 2) % 5]);
  }
  a[0] ^= rc;
#endif
}

// Full 24-round permutation.  UNROLL rounds per loop iteration (a tuning knob:
// more unrolling gives the scheduler more independent work at a larger code size).
template <int UNROLL = 2>
__host__ __device__ __forceinline__ void keccak_f1600(uint64_t (&a)[25]) {
#if defined(__CUDA_ARCH__)
#pragma unroll 1
  for (int r = 0; r < 24; r += UNROLL) {
#pragma unroll
    for (int k = 0; k < UNROLL; k++) keccak_round(a, kKeccakRC[r + k]);
  }
#else
  for (int r = 0; r < 24; r++) keccak_round(a, kKeccakRC[r]);
#endif
}

// Sponge padding constants for one 136-byte block (rate of SHA3-256).
static constexpr int kRateLanes = 17;
static constexpr uint64_t kPadEnd = 0x8000000000000000ULL;  // 0x80 at byte 135 (lane 16)

// SHA3-256 (suffix 0x06) of a message of 2 lanes = one 16-byte QM31 leaf.
__host__ __device__ __forceinline__ void sha3_16(uint64_t l0, uint64_t l1, uint64_t (&out)[4], uint64_t suffix = 0x06) {
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; i++) a[i] = 0;
  a[0] = l0;
  a[1] = l1;
  a[2] = suffix;
  a[16] = kPadEnd;
  keccak_f1600(a);
#pragma unroll
  for (int i = 0; i < 4; i++) out[i] = a[i];
}

// SHA3-256 of the 64-byte concatenation left || right (Merkle parent).
__host__ __device__ __forceinline__ void sha3_pair(const uint64_t (&l)[4], const uint64_t (&r)[4], uint64_t (&out)[4]) {
  uint64_t a[25];
#pragma unroll
  for (int i = 0; i < 25; i++) a[i] = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) { a[i] = l[i]; a[4 + i] = r[i]; }
  a[8] = 0x06;
  a[16] = kPadEnd;
  keccak_f1600(a);
#pragma unroll
  for (int i = 0; i < 4; i++) out[i] = a[i];
}

}  // namespace azk
