// Host-compiled check of the CUDA library's __host__ __device__ helpers
// (apple_b200/csrc/*.cuh) against the CPU oracle.  Built and run by
// tests/test_device_helpers_on_host.py; exits non-zero on the first mismatch.
#include <cstdio>
#include <random>

#include "azk_oracle.hpp"
#include "azk_field.cuh"
#include "azk_keccak.cuh"
#include "azk_transcript.cuh"

namespace O = azk_oracle;

static int fails = 0;
#define CHECK(c, ...)                      \
  do {                                     \
    if (!(c)) {                            \
      std::fprintf(stderr, __VA_ARGS__);   \
      std::fprintf(stderr, "\n");          \
      if (++fails > 10) return 1;          \
    }                                      \
  } while (0)

int main() {
  std::mt19937_64 rng(12345);
  // Keccak-f[1600]
  for (int t = 0; t < 200; t++) {
    uint64_t a[25], b[25];
    for (int i = 0; i < 25; i++) a[i] = b[i] = rng();
    azk::keccak_f1600(a);
    O::keccak_f1600(b);
    for (int i = 0; i < 25; i++) CHECK(a[i] == b[i], "keccak lane %d mismatch", i);
  }
  // SHA3 of 16-byte leaves and 64-byte pairs
  for (int t = 0; t < 200; t++) {
    uint8_t m[64];
    for (auto& x : m) x = (uint8_t)rng();
    uint64_t l[8];
    std::memcpy(l, m, 64);
    uint64_t d[4];
    azk::sha3_16(l[0], l[1], d);
    O::Digest e = O::sha3_256(m, 16);
    CHECK(std::memcmp(d, e.b, 32) == 0, "sha3_16 mismatch");
    uint64_t L[4] = {l[0], l[1], l[2], l[3]}, R[4] = {l[4], l[5], l[6], l[7]};
    azk::sha3_pair(L, R, d);
    e = O::sha3_256(m, 64);
    CHECK(std::memcmp(d, e.b, 32) == 0, "sha3_pair mismatch");
  }
  // Fields
  std::uniform_int_distribution<uint32_t> U(0, O::m31::P - 1);
  for (int t = 0; t < 20000; t++) {
    uint32_t x = U(rng), y = U(rng);
    if (t < 8) { x = (t & 1) ? 0 : O::m31::P - 1; y = (t & 2) ? 0 : O::m31::P - 1; }
    CHECK(azk::m31_mul(x, y) == O::m31::mul(x, y), "m31 mul");
    CHECK(azk::m31_mul_dbl(x, y << 1) == O::m31::mul(x, y), "m31 mul by a doubled operand");
    CHECK(azk::m31_mul_dbl(O::m31::P, y << 1) == 0, "m31 mul by a doubled operand, redundant zero");
    CHECK(azk::m31_add(x, y) == O::m31::add(x, y), "m31 add");
    CHECK(azk::m31_sub(x, y) == O::m31::sub(x, y), "m31 sub");
    CHECK(azk::m31_half(x) == O::m31::mul(x, 1073741824u), "m31 half");
    azk::qm31 a{U(rng), U(rng), U(rng), U(rng)}, b{U(rng), U(rng), U(rng), U(rng)}, c{U(rng), U(rng), U(rng), U(rng)};
    O::QM31 A{a.a, a.b, a.c, a.d}, B{b.a, b.b, b.c, b.d}, C{c.a, c.b, c.c, c.d};
    azk::qm31 r = azk::q_mul(a, b);
    O::QM31 R = O::q_mul(A, B);
    CHECK(r.a == R.a && r.b == R.b && r.c == R.c && r.d == R.d, "qm31 mul");
    uint32_t tw = U(rng) | 1;
    azk::qm31 f = azk::fri_fold_pair(a, b, tw, c);
    O::QM31 F = O::fold_pair(A, B, O::QM31{tw, 0, 0, 0}, C);
    CHECK(f.a == F.a && f.b == F.b && f.c == F.c && f.d == F.d, "fold pair");
  }
  for (int t = 0; t < 200; t++) {
    uint32_t x = U(rng) | 1;
    CHECK(azk::m31_mul(azk::m31_inv(x), x) == 1, "m31 inv");
  }
  // Circle points of the canonical domain, all natural indices of small domains
  for (uint32_t logN = 1; logN <= 12; logN++) {
    O::Domain d = O::canonical_domain(logN);
    for (uint32_t i = 0; i < (1u << logN); i++) {
      uint32_t idx = azk::circle_point_index(logN, i);
      CHECK(idx == O::domain_point_index(d, i), "point index log %u i %u", logN, i);
      azk::cpoint p = azk::cp_from_index(idx);
      O::Point q = O::index_to_point(idx);
      CHECK(p.x == q.x && p.y == q.y, "point log %u i %u", logN, i);
    }
    for (uint32_t i = 0; i < (1u << logN); i++) CHECK(azk::bit_reverse(i, logN) == O::bit_reverse(i, logN), "bitrev");
  }
  // Transcript: random frames and the circle round frames
  for (int t = 0; t < 50; t++) {
    azk::Transcript T;
    azk::tr_reset(T);
    O::Transcript OT;
    for (int f = 0; f < 4; f++) {
      std::vector<uint8_t> msg(rng() % 300);
      for (auto& x : msg) x = (uint8_t)rng();
      azk::tr_absorb(T, msg.data(), (uint32_t)msg.size());
      OT.absorb(msg.data(), msg.size());
    }
    for (int i = 0; i < 25; i++) CHECK(T.st[i] == OT.st[i], "transcript state");
    uint32_t w[80];
    azk::tr_squeeze_u32(T, 80, 1u << 20 | 7, w);
    auto ow = OT.squeeze_u32(80, 1u << 20 | 7);
    for (int i = 0; i < 80; i++) CHECK(w[i] == ow[i], "squeeze word %d", i);
    uint64_t root[4] = {rng(), rng(), rng(), rng()};
    O::Digest od;
    std::memcpy(od.b, root, 32);
    uint32_t ch[4];
    azk::circle_round(T, (uint32_t)t, root, ch);
    O::QM31 oc = O::transcript_round(OT, (uint32_t)t, od);
    CHECK(ch[0] == oc.a && ch[1] == oc.b && ch[2] == oc.c && ch[3] == oc.d, "circle round challenge");
  }
  if (fails) return 1;
  std::printf("host check ok\n");
  return 0;
}
