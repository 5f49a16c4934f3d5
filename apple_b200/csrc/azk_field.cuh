// M31 / CM31 / QM31 arithmetic for sm_100a (and the host, for unit tests).
//
// M31 products are 32x32->64 integer multiplies followed by a Mersenne fold
// (v & p) + (v >> 31); every function returns the canonical representative in
// [0, p), so results equal the reference's CPU oracle (SumcheckOracle.swift:3-147,
// CM31Field.swift:30-96, QM31Field.swift:36-139) bit for bit.  QM31 = CM31[u] with
// u^2 = 2 + i, stored as four little-endian u32 limbs (a, b, c, d).
#pragma once
#include <stdint.h>
#include "azk_keccak.cuh"

namespace azk {

static constexpr uint32_t kP = 2147483647u;
static constexpr uint32_t kInv2 = 1073741824u;

// s < 2p -> s mod p.  s - p is below s exactly when s >= p (otherwise it wraps
// above it), so the reduction is an unsigned minimum: one subtract, one min.
__host__ __device__ __forceinline__ uint32_t m31_reduce_once(uint32_t s) {
  const uint32_t t = s - kP;
  return t < s ? t : s;
}
__host__ __device__ __forceinline__ uint32_t m31_fold64(uint64_t v) {
  // v < 2^62: two Mersenne folds then one conditional subtraction
  uint64_t r = (v & kP) + (v >> 31);
  uint32_t s = (uint32_t)((r & kP) + (r >> 31));
  return s >= kP ? s - kP : s;
}
// Inputs are at most p (canonical values, or p itself as a redundant zero).
__host__ __device__ __forceinline__ uint32_t m31_add(uint32_t a, uint32_t b) { return m31_reduce_once(a + b); }
// a + (p - b) lies in [0, 2p): one reduction, no branch on a >= b.
__host__ __device__ __forceinline__ uint32_t m31_sub(uint32_t a, uint32_t b) { return m31_reduce_once(a + (kP - b)); }
__host__ __device__ __forceinline__ uint32_t m31_neg(uint32_t a) { return a == 0 ? 0 : kP - a; }
// a, b <= p: the product is below 2^62 - 2^32 + 2, so one Mersenne fold of it in
// 32-bit arithmetic, (v mod 2^31) + (v >> 31), is below 2p and one reduction
// finishes it.
__host__ __device__ __forceinline__ uint32_t m31_mul(uint32_t a, uint32_t b) {
  const uint64_t v = (uint64_t)a * (uint64_t)b;
  return m31_reduce_once(((uint32_t)v & kP) + (uint32_t)(v >> 31));
}
// a * t for a <= p and t2 = 2t (t < p): the 64-bit product a t2 = 2 a t has a t >> 31
// in its high word and (a t mod 2^31) << 1 in its low word, so the Mersenne fold is
// hi + (lo >> 1) (below 2p), without masking the low word.
__host__ __device__ __forceinline__ uint32_t m31_mul_dbl(uint32_t a, uint32_t t2) {
  const uint64_t v = (uint64_t)a * (uint64_t)t2;
  return m31_reduce_once((uint32_t)(v >> 32) + ((uint32_t)v >> 1));
}
// x * 2^-1 mod p: halve an even value, or (x + p) / 2 = (x >> 1) + 2^30 for an odd one.
__host__ __device__ __forceinline__ uint32_t m31_half(uint32_t a) { return (a >> 1) + ((a & 1u) << 30); }
__host__ __device__ __forceinline__ uint32_t m31_pow(uint32_t b, uint32_t e) {
  uint32_t r = 1;
  while (e) {
    if (e & 1u) r = m31_mul(r, b);
    e >>= 1;
    b = m31_mul(b, b);
  }
  return r;
}
// Fermat inverse a^(p-2); returns 0 for a == 0 (callers validate).
__host__ __device__ __forceinline__ uint32_t m31_inv(uint32_t a) { return m31_pow(a, kP - 2); }

struct qm31 {
  uint32_t a, b, c, d;
};

__host__ __device__ __forceinline__ qm31 q_add(qm31 x, qm31 y) { return {m31_add(x.a, y.a), m31_add(x.b, y.b), m31_add(x.c, y.c), m31_add(x.d, y.d)}; }
__host__ __device__ __forceinline__ qm31 q_sub(qm31 x, qm31 y) { return {m31_sub(x.a, y.a), m31_sub(x.b, y.b), m31_sub(x.c, y.c), m31_sub(x.d, y.d)}; }
__host__ __device__ __forceinline__ qm31 q_mul_m31(qm31 x, uint32_t s) { return {m31_mul(x.a, s), m31_mul(x.b, s), m31_mul(x.c, s), m31_mul(x.d, s)}; }
__host__ __device__ __forceinline__ qm31 q_half(qm31 x) { return {m31_half(x.a), m31_half(x.b), m31_half(x.c), m31_half(x.d)}; }

// CM31 product (re, im) = (ac - bd, ad + bc), each term reduced as in the reference.
__host__ __device__ __forceinline__ void cm_mul(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t& re, uint32_t& im) {
  re = m31_sub(m31_mul(a, c), m31_mul(b, d));
  im = m31_add(m31_mul(a, d), m31_mul(b, c));
}
// QM31 product: (x0 + x1 u)(y0 + y1 u) = x0 y0 + (2+i) x1 y1 + (x0 y1 + x1 y0) u
__host__ __device__ __forceinline__ qm31 q_mul(qm31 x, qm31 y) {
  uint32_t acr, aci, bdr, bdi, adr, adi, bcr, bci;
  cm_mul(x.a, x.b, y.a, y.b, acr, aci);
  cm_mul(x.c, x.d, y.c, y.d, bdr, bdi);
  cm_mul(x.a, x.b, y.c, y.d, adr, adi);
  cm_mul(x.c, x.d, y.a, y.b, bcr, bci);
  // (2 + i)(r + i s) = (2r - s) + i(2s + r); field arithmetic is exact, so adds
  // stand in for the reference's multiplications by 2 and 1 with equal results.
  uint32_t nr = m31_sub(m31_add(bdr, bdr), bdi);
  uint32_t ni = m31_add(m31_add(bdi, bdi), bdr);
  return {m31_add(acr, nr), m31_add(aci, ni), m31_add(adr, bcr), m31_add(adi, bci)};
}

// One FRI fold of the pair (pos, neg) with inverse-domain value t (an M31) and
// challenge ch: ((pos + neg) + ch * ((pos - neg) * t)) / 2  (QM31FRIFold.swift:30-41).
__host__ __device__ __forceinline__ qm31 fri_fold_pair(qm31 pos, qm31 neg, uint32_t t, qm31 ch) {
  qm31 even = q_add(pos, neg);
  qm31 odd = q_mul_m31(q_sub(pos, neg), t);
  return q_half(q_add(even, q_mul(ch, odd)));
}

// ---- circle group over M31 (CircleDomain.swift:3-101) ----
struct cpoint {
  uint32_t x, y;
};
__host__ __device__ __forceinline__ cpoint cp_add(cpoint p, cpoint q) {
  return {m31_sub(m31_mul(p.x, q.x), m31_mul(p.y, q.y)), m31_add(m31_mul(p.x, q.y), m31_mul(p.y, q.x))};
}
// generator^k with the M31 circle generator (2, 1268011823)
__host__ __device__ __forceinline__ cpoint cp_from_index(uint32_t k) {
  cpoint r = {1, 0}, p = {2, 1268011823u};
  while (k) {
    if (k & 1u) r = cp_add(r, p);
    k >>= 1;
    p = cp_add(p, p);
  }
  return r;
}
__host__ __device__ __forceinline__ uint32_t double_x(uint32_t x) {
  uint32_t s = m31_mul(x, x);
  return m31_sub(m31_add(s, s), 1);
}
__host__ __device__ __forceinline__ uint32_t bit_reverse(uint32_t i, uint32_t bits) {
#if defined(__CUDA_ARCH__)
  return bits ? (__brev(i) >> (32 - bits)) : 0;
#else
  uint32_t r = 0;
  for (uint32_t k = 0; k < bits; k++) { r = (r << 1) | (i & 1u); i >>= 1; }
  return r;
#endif
}
// Point index of natural-order element i of the canonical domain of size 2^logN
// (CircleDomain.swift:225-239, 273-285): half coset halfOdds(logN-1) and its conjugate.
__host__ __device__ __forceinline__ uint32_t circle_point_index(uint32_t logN, uint32_t i) {
  const uint32_t mask = 0x7FFFFFFFu;
  uint32_t initial = (uint32_t)((1ull << (31 - (logN + 1))) & mask);
  uint32_t step = (uint32_t)((1ull << (31 - (logN - 1))) & mask);
  uint32_t half = 1u << (logN - 1);
  uint32_t off = i < half ? i : i - half;
  uint32_t idx = (uint32_t)(((uint64_t)initial + (uint64_t)step * off) & mask);
  if (i >= half) idx = (uint32_t)((0x80000000ull - idx) & mask);
  return idx;
}

}  // namespace azk
