// azk_oracle.hpp -- CPU ORACLE (test infrastructure only).
//
// A C++17 restatement of the CPU oracles of AppleZKProver (Swift) for the
// commit-and-fold superstep: Keccak-f[1600]/SHA3-256/Keccak-256, the sponge
// transcript, the SHA3 Merkle tree, M31/CM31/QM31 arithmetic, the circle domain
// and its twiddles, the Circle FFT codeword, QM31/Circle FRI folding, the Circle
// FRI transcript V1, the PCS proof builder/codec/verifier and the M31 sum-check
// oracles.  Every function names the reference file:line it follows.
//
// This header is the CHECKER.  Only tests/, __graft_entry__.smoke() and the
// bench's cpu_baseline / reference arm use it.  The CUDA library never includes
// or links it.
//
// Where the reference recomputes something from scratch for every call (the O(R^2)
// prefix-transcript replay in the proof builder, the full Merkle rebuild per
// opening), this oracle keeps the same outputs but builds each tree once and
// carries the transcript forward; `literal` variants reproduce the reference's
// recomputation for small sizes so a test can show both agree byte for byte.
#pragma once
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include <array>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace azk_oracle {

using u8 = uint8_t;
using u32 = uint32_t;
using u64 = uint64_t;
using Bytes = std::vector<u8>;

// Error kinds mirror AppleZKProverError (MetalTypes.swift:3-22).
enum class Err : int {
  ok = 0,
  invalidInputLayout = 1,
  invalidLeafCount = 2,
  unsupportedOneBlockLength = 3,
  invalidPrehashedLeafLength = 4,
  correctnessValidationFailed = 5,
};

struct OracleError : std::runtime_error {
  Err kind;
  long long value;
  OracleError(Err k, const std::string& m, long long v = 0) : std::runtime_error(m), kind(k), value(v) {}
};
[[noreturn]] inline void fail(Err k = Err::invalidInputLayout, const char* m = "invalid input layout", long long v = 0) {
  throw OracleError(k, m, v);
}
inline void require(bool c, Err k = Err::invalidInputLayout, const char* m = "invalid input layout", long long v = 0) {
  if (!c) fail(k, m, v);
}

// ---------------------------------------------------------------------------
// Little-endian byte helpers (CanonicalBinary, CircleProofFormat.swift:1766-1787)
// ---------------------------------------------------------------------------
inline void put_u32(Bytes& d, u32 v) { for (int i = 0; i < 4; i++) d.push_back(u8(v >> (8 * i))); }
inline void put_u64(Bytes& d, u64 v) { for (int i = 0; i < 8; i++) d.push_back(u8(v >> (8 * i))); }
inline void put_bytes(Bytes& d, const Bytes& s) { d.insert(d.end(), s.begin(), s.end()); }
inline void put_str(Bytes& d, const char* s) { d.insert(d.end(), s, s + std::strlen(s)); }
inline u32 get_u32(const u8* p) { return u32(p[0]) | u32(p[1]) << 8 | u32(p[2]) << 16 | u32(p[3]) << 24; }
inline u64 get_u64(const u8* p) { return u64(get_u32(p)) | u64(get_u32(p + 4)) << 32; }

inline bool is_pow2(u64 v) { return v && !(v & (v - 1)); }
inline int log2_floor(u64 v) { int r = 0; if (v < 1) v = 1; while (v > 1) { v >>= 1; r++; } return r; }

// ---------------------------------------------------------------------------
// Keccak-f[1600]  (SHA3Oracle.swift:102-135 constants, :242-280 permutation)
// ---------------------------------------------------------------------------
static const u64 kRC[24] = {
    0x0000000000000001ULL, 0x0000000000008082ULL, 0x800000000000808AULL, 0x8000000080008000ULL,
    0x000000000000808BULL, 0x0000000080000001ULL, 0x8000000080008081ULL, 0x8000000000008009ULL,
    0x000000000000008AULL, 0x0000000000000088ULL, 0x0000000080008009ULL, 0x000000008000000AULL,
    0x000000008000808BULL, 0x800000000000008BULL, 0x8000000000008089ULL, 0x8000000000008003ULL,
    0x8000000000008002ULL, 0x8000000000000080ULL, 0x000000000000800AULL, 0x800000008000000AULL,
    0x8000000080008081ULL, 0x8000000000008080ULL, 0x0000000080000001ULL, 0x8000000080008008ULL};
static const int kRho[24] = {1, 3, 6, 10, 15, 21, 28, 36, 45, 55, 2, 14, 27, 41, 56, 8, 25, 43, 62, 18, 39, 61, 20, 44};
static const int kPi[24] = {10, 7, 11, 17, 18, 3, 5, 16, 8, 21, 24, 4, 15, 23, 19, 13, 12, 2, 20, 14, 22, 9, 6, 1};

inline u64 rotl64(u64 v, int n) { n &= 63; return n ? (v << n) | (v >> (64 - n)) : v; }

inline void keccak_f1600(u64 s[25]) {
  for (int round = 0; round < 24; round++) {
    u64 c[5];
    for (int x = 0; x < 5; x++) c[x] = s[x] ^ s[x + 5] ^ s[x + 10] ^ s[x + 15] ^ s[x + 20];
    for (int x = 0; x < 5; x++) {
      u64 d = c[(x + 4) % 5] ^ rotl64(c[(x + 1) % 5], 1);
      for (int y = 0; y < 25; y += 5) s[x + y] ^= d;
    }
    u64 cur = s[1];
    for (int i = 0; i < 24; i++) {
      int dst = kPi[i];
      u64 nxt = s[dst];
      s[dst] = rotl64(cur, kRho[i]);
      cur = nxt;
    }
    for (int row = 0; row < 25; row += 5) {
      u64 b[5];
      for (int x = 0; x < 5; x++) b[x] = s[row + x];
      for (int x = 0; x < 5; x++) s[row + x] = b[x] ^ (~b[(x + 1) % 5] & b[(x + 2) % 5]);
    }
    s[0] ^= kRC[round];
  }
}

// XOR `rate` bytes (little-endian lanes) into the state (SHA3Oracle.swift:225-240).
inline void absorb_block(u64 s[25], const u8* p, size_t rate) {
  for (size_t lane = 0; lane < rate / 8; lane++) {
    u64 v = 0;
    for (int k = 0; k < 8; k++) v |= u64(p[lane * 8 + k]) << (8 * k);
    s[lane] ^= v;
  }
}

// Generic sponge (SHA3Oracle.swift:181-219).
inline void sponge(const u8* data, size_t len, size_t rate, u8 suffix, u8* out, size_t outLen) {
  require(rate > 0 && rate <= 200 && rate % 8 == 0);
  u64 s[25] = {0};
  size_t off = 0;
  while (off + rate <= len) { absorb_block(s, data + off, rate); keccak_f1600(s); off += rate; }
  u8 tail[200] = {0};
  size_t tc = len - off;
  if (tc) std::memcpy(tail, data + off, tc);
  tail[tc] ^= suffix;
  tail[rate - 1] ^= 0x80;
  absorb_block(s, tail, rate);
  keccak_f1600(s);
  size_t produced = 0;
  while (produced < outLen) {
    size_t take = std::min(rate, outLen - produced);
    for (size_t b = 0; b < take; b++) out[produced + b] = u8(s[b >> 3] >> (8 * (b & 7)));
    produced += take;
    if (produced < outLen) keccak_f1600(s);
  }
}

static const size_t kSha3Rate = 136;  // SHA3Oracle.swift:4

struct Digest { u8 b[32]; bool operator==(const Digest& o) const { return std::memcmp(b, o.b, 32) == 0; } };

inline Digest sha3_256(const u8* d, size_t n) { Digest r; sponge(d, n, kSha3Rate, 0x06, r.b, 32); return r; }
inline Digest sha3_256(const Bytes& d) { return sha3_256(d.data(), d.size()); }
inline Digest keccak_256(const u8* d, size_t n) { Digest r; sponge(d, n, kSha3Rate, 0x01, r.b, 32); return r; }
inline Digest sha3_pair(const Digest& l, const Digest& r) {
  u8 buf[64];
  std::memcpy(buf, l.b, 32);
  std::memcpy(buf + 32, r.b, 32);
  return sha3_256(buf, 64);
}

// ---------------------------------------------------------------------------
// Sponge transcript (SHA3Oracle.TranscriptState, SHA3Oracle.swift:8-98).
// absorb() pads and permutes on every call; squeeze*() copy the state.
// ---------------------------------------------------------------------------
struct Transcript {
  u64 st[25];
  Transcript() { reset(); }
  void reset() { std::memset(st, 0, sizeof(st)); }
  void absorb(const u8* p, size_t n, u8 suffix = 0x06) {
    size_t off = 0;
    while (off + kSha3Rate <= n) { absorb_block(st, p + off, kSha3Rate); keccak_f1600(st); off += kSha3Rate; }
    u8 tail[kSha3Rate] = {0};
    size_t tc = n - off;
    if (tc) std::memcpy(tail, p + off, tc);
    tail[tc] ^= suffix;
    tail[kSha3Rate - 1] ^= 0x80;
    absorb_block(st, tail, kSha3Rate);
    keccak_f1600(st);
  }
  void absorb(const Bytes& b) { absorb(b.data(), b.size()); }
  void absorb(const Digest& d) { absorb(d.b, 32); }
  // SHA3Oracle.swift:41-70
  std::vector<u32> squeeze_u32(size_t count, u32 modulus) const {
    require(modulus > 0);
    const size_t wordsPerBlock = kSha3Rate / 4;  // 34
    const u64 space = u64(1) << 32;
    const u64 limit = space - (space % modulus);
    u64 s[25];
    std::memcpy(s, st, sizeof(s));
    std::vector<u32> out;
    out.reserve(count);
    size_t idx = 0;
    while (out.size() < count) {
      if (idx > 0 && idx % wordsPerBlock == 0) keccak_f1600(s);
      size_t w = idx % wordsPerBlock;
      u64 cand = u32(s[w >> 1] >> ((w & 1) * 32));
      idx++;
      if (cand < limit) out.push_back(u32(cand % modulus));
    }
    return out;
  }
  // SHA3Oracle.swift:72-97
  Bytes squeeze_bytes(size_t count) const {
    u64 s[25];
    std::memcpy(s, st, sizeof(s));
    Bytes out;
    size_t bi = 0;
    while (out.size() < count) {
      if (bi > 0 && bi % kSha3Rate == 0) keccak_f1600(s);
      size_t lane = (bi % kSha3Rate) >> 3, lb = (bi % kSha3Rate) & 7;
      out.push_back(u8(s[lane] >> (8 * lb)));
      bi++;
    }
    return out;
  }
};

// ---------------------------------------------------------------------------
// M31 / CM31 / QM31 (SumcheckOracle.swift:3-147, CM31Field.swift:30-96,
// QM31Field.swift:36-139, CircleCodeword.swift:266-279)
// ---------------------------------------------------------------------------
namespace m31 {
static const u32 P = 2147483647u;
inline u32 reduce(u64 v) {  // SumcheckOracle.swift:140-146
  const u64 m = P;
  u64 r = (v & m) + (v >> 31);
  r = (r & m) + (r >> 31);
  r = (r & m) + (r >> 31);
  return u32(r >= m ? r - m : r);
}
inline u32 add(u32 a, u32 b) { u32 s = a + b; return s >= P ? s - P : s; }
inline u32 sub(u32 a, u32 b) { return a >= b ? a - b : P - (b - a); }
inline u32 neg(u32 a) { return a == 0 ? 0 : P - a; }
inline u32 mul(u32 a, u32 b) { return reduce(u64(a) * u64(b)); }
inline u32 sqr(u32 a) { return mul(a, a); }
inline u32 pow(u32 b, u32 e) {
  u32 r = 1, p = b;
  while (e) { if (e & 1) r = mul(r, p); e >>= 1; if (e) p = sqr(p); }
  return r;
}
inline u32 inv(u32 a) { require(a > 0 && a < P); return pow(a, P - 2); }
inline void batch_inverse(const u32* in, u32* out, size_t n) {  // SumcheckOracle.swift:42-63
  if (!n) return;
  std::vector<u32> pre(n);
  u32 acc = 1;
  for (size_t i = 0; i < n; i++) { require(in[i] != 0 && in[i] < P); pre[i] = acc; acc = mul(acc, in[i]); }
  u32 ia = inv(acc);
  for (size_t i = n; i-- > 0;) { u32 v = in[i]; out[i] = mul(ia, pre[i]); ia = mul(ia, v); }
}
}  // namespace m31

struct CM31 { u32 re, im; };
inline CM31 cm_add(CM31 a, CM31 b) { return {m31::add(a.re, b.re), m31::add(a.im, b.im)}; }
inline CM31 cm_sub(CM31 a, CM31 b) { return {m31::sub(a.re, b.re), m31::sub(a.im, b.im)}; }
inline CM31 cm_neg(CM31 a) { return {m31::neg(a.re), m31::neg(a.im)}; }
inline CM31 cm_mul(CM31 a, CM31 b) {  // CM31Field.swift:61-71
  u32 ac = m31::mul(a.re, b.re), bd = m31::mul(a.im, b.im), ad = m31::mul(a.re, b.im), bc = m31::mul(a.im, b.re);
  return {m31::sub(ac, bd), m31::add(ad, bc)};
}
inline CM31 cm_sqr(CM31 a) {  // CM31Field.swift:73-80
  u32 re = m31::sub(m31::sqr(a.re), m31::sqr(a.im));
  u32 cr = m31::mul(a.re, a.im);
  return {re, m31::add(cr, cr)};
}
inline CM31 cm_inv(CM31 a) {  // CM31Field.swift:82-96
  require(a.re < m31::P && a.im < m31::P && (a.re || a.im));
  u32 den = m31::add(m31::sqr(a.re), m31::sqr(a.im));
  u32 di = m31::inv(den);
  return {m31::mul(a.re, di), m31::mul(m31::neg(a.im), di)};
}

struct QM31 {
  u32 a, b, c, d;
  bool operator==(const QM31& o) const { return a == o.a && b == o.b && c == o.c && d == o.d; }
  bool operator!=(const QM31& o) const { return !(*this == o); }
};
static const CM31 kNonResidue = {2, 1};  // QM31Field.swift:37
inline CM31 q_c0(QM31 x) { return {x.a, x.b}; }
inline CM31 q_c1(QM31 x) { return {x.c, x.d}; }
inline QM31 q_make(CM31 c0, CM31 c1) { return {c0.re, c0.im, c1.re, c1.im}; }
inline bool q_is_zero(QM31 x) { return !x.a && !x.b && !x.c && !x.d; }
inline bool q_canonical(QM31 x) { return x.a < m31::P && x.b < m31::P && x.c < m31::P && x.d < m31::P; }
inline QM31 q_add(QM31 x, QM31 y) { return q_make(cm_add(q_c0(x), q_c0(y)), cm_add(q_c1(x), q_c1(y))); }
inline QM31 q_sub(QM31 x, QM31 y) { return q_make(cm_sub(q_c0(x), q_c0(y)), cm_sub(q_c1(x), q_c1(y))); }
inline QM31 q_neg(QM31 x) { return q_make(cm_neg(q_c0(x)), cm_neg(q_c1(x))); }
inline QM31 q_mul(QM31 x, QM31 y) {  // QM31Field.swift:80-90
  CM31 ac = cm_mul(q_c0(x), q_c0(y)), bd = cm_mul(q_c1(x), q_c1(y));
  CM31 ad = cm_mul(q_c0(x), q_c1(y)), bc = cm_mul(q_c1(x), q_c0(y));
  return q_make(cm_add(ac, cm_mul(kNonResidue, bd)), cm_add(ad, bc));
}
inline QM31 q_mul_m31(QM31 x, u32 s) {  // CircleCodeword.swift:266-279
  return {m31::mul(x.a, s), m31::mul(x.b, s), m31::mul(x.c, s), m31::mul(x.d, s)};
}
inline QM31 q_inv(QM31 x) {  // QM31Field.swift:102-117
  require(q_canonical(x) && !q_is_zero(x));
  CM31 aa = cm_sqr(q_c0(x)), bb = cm_sqr(q_c1(x));
  CM31 den = cm_sub(aa, cm_mul(kNonResidue, bb));
  CM31 di = cm_inv(den);
  return q_make(cm_mul(q_c0(x), di), cm_mul(cm_neg(q_c1(x)), di));
}
static const QM31 kInverseTwo = {1073741824u, 0, 0, 0};  // QM31FRIFold.swift:4-9

inline void put_qm31(Bytes& d, QM31 v) { put_u32(d, v.a); put_u32(d, v.b); put_u32(d, v.c); put_u32(d, v.d); }
inline QM31 get_qm31(const u8* p) { return {get_u32(p), get_u32(p + 4), get_u32(p + 8), get_u32(p + 12)}; }
inline Bytes pack_qm31(const std::vector<QM31>& v) {  // QM31CanonicalEncoding.pack, CircleProofFormat.swift:6-22
  Bytes d;
  d.reserve(v.size() * 16);
  for (auto& x : v) put_qm31(d, x);
  return d;
}

// ---------------------------------------------------------------------------
// Circle group over M31 (CircleDomain.swift:3-185)
// ---------------------------------------------------------------------------
struct Point { u32 x, y; bool operator==(const Point& o) const { return x == o.x && y == o.y; } };
static const Point kGenerator = {2, 1268011823u};  // CircleDomain.swift:5
static const Point kIdentity = {1, 0};
inline Point pt_add(Point p, Point q) {  // CircleDomain.swift:32-41
  u32 xx = m31::mul(p.x, q.x), yy = m31::mul(p.y, q.y), xy = m31::mul(p.x, q.y), yx = m31::mul(p.y, q.x);
  return {m31::sub(xx, yy), m31::add(xy, yx)};
}
inline Point pt_double(Point p) { return pt_add(p, p); }
inline Point pt_mul(Point p, u64 k) {  // CircleDomain.swift:43-56
  Point r = kIdentity, pw = p;
  while (k) { if (k & 1) r = pt_add(r, pw); k >>= 1; if (k) pw = pt_double(pw); }
  return r;
}
inline Point pt_conj(Point p) { return {p.x, m31::neg(p.y)}; }
static const u32 kCircleLogOrder = 31;
static const u32 kCircleOrderMask = 0x7FFFFFFFu;
inline Point index_to_point(u32 idx) { return pt_mul(kGenerator, idx); }  // CircleDomain.swift:99-101
inline u32 subgroup_generator_index(u32 logSize) {  // CircleDomain.swift:73-78 (index reduced mod 2^31)
  return u32((u64(1) << (kCircleLogOrder - logSize)) & kCircleOrderMask);
}
inline u32 double_x(u32 x) { return m31::sub(m31::add(m31::sqr(x), m31::sqr(x)), 1); }  // CircleDomain.swift:339-341
inline void validate_point(Point p) {  // CircleDomain.swift:265-271
  require(p.x < m31::P && p.y < m31::P);
  require(m31::add(m31::sqr(p.x), m31::sqr(p.y)) == 1);
}

inline u64 bit_reverse(u64 i, u32 logSize) {  // CircleDomain.swift:325-336
  u64 r = 0;
  for (u32 k = 0; k < logSize; k++) { r = (r << 1) | (i & 1); i >>= 1; }
  return r;
}

// Canonical bit-reversed circle domain (CircleDomain.swift:187-262).
struct Domain {
  u32 logSize = 0;
  u32 halfCosetInitial = 0;  // index of the half-coset's first point
  u32 halfCosetLogSize = 0;
  u32 storageOrder = 1;      // 0 natural, 1 bit-reversed, 2 coset-natural
  u64 size() const { return u64(1) << logSize; }
  u64 half() const { return size() >> 1; }
  bool canonical() const {  // CircleDomain.swift:254-261
    u32 step = subgroup_generator_index(halfCosetLogSize);
    u32 four = u32((u64(halfCosetInitial) * 4) & kCircleOrderMask);
    return four == step;
  }
};
inline Domain canonical_domain(u32 logSize, u32 storageOrder = 1) {
  require(logSize >= 1 && logSize <= 30);
  Domain d;
  d.logSize = logSize;
  d.halfCosetLogSize = logSize - 1;
  d.halfCosetInitial = subgroup_generator_index(logSize + 1);  // halfOdds(logSize-1): generator of order 2^(logSize+1)
  d.storageOrder = storageOrder;
  return d;
}
// Point index of natural-order domain element i (CircleDomain.swift:273-285).
inline u32 domain_point_index(const Domain& d, u64 i) {
  require(i < d.size());
  u32 step = subgroup_generator_index(d.halfCosetLogSize);
  u64 h = d.half();
  u64 off = i < h ? i : i - h;
  u32 idx = u32((u64(d.halfCosetInitial) + u64(step) * (off & kCircleOrderMask)) & kCircleOrderMask);
  if (i >= h) idx = u32((u64(1) << 31) - idx) & kCircleOrderMask;
  return idx;
}
inline u64 coset_to_circle_index(u64 ci, u32 logSize) {  // CircleDomain.swift:351-356
  if (ci % 2 == 0) return ci / 2;
  return ((u64(2) << logSize) - ci) / 2;
}
inline u64 circle_to_coset_index(u64 i, u32 logSize) {  // CircleDomain.swift:343-349
  u64 n = u64(1) << logSize;
  if (i < n / 2) return i * 2;
  return (n - 1 - i) * 2 + 1;
}
inline u64 natural_from_storage(const Domain& d, u64 s) {  // CircleDomain.swift:303-323
  require(s < d.size());
  if (d.storageOrder == 0) return s;
  if (d.storageOrder == 1) return bit_reverse(s, d.logSize);
  return coset_to_circle_index(s, d.logSize);
}
inline Point domain_point(const Domain& d, u64 natural) { return index_to_point(domain_point_index(d, natural)); }

// All natural-order points, computed by repeated addition (equal to generator^index
// by the group homomorphism; the second half is the conjugate of the first).
inline std::vector<Point> natural_points(const Domain& d) {
  u64 h = d.half();
  std::vector<Point> pts(d.size());
  Point p0 = index_to_point(d.halfCosetInitial);
  Point step = index_to_point(subgroup_generator_index(d.halfCosetLogSize));
  const int T = 64;
  u64 chunk = (h + T - 1) / T;
#pragma omp parallel for schedule(static)
  for (int t = 0; t < T; t++) {
    u64 lo = u64(t) * chunk, hi = std::min(h, lo + chunk);
    if (lo >= hi) continue;
    Point p = pt_add(p0, pt_mul(step, lo));
    for (u64 i = lo; i < hi; i++) { pts[i] = p; pts[i + h] = pt_conj(p); p = pt_add(p, step); }
  }
  return pts;
}
inline std::vector<Point> storage_points(const Domain& d) {
  auto nat = natural_points(d);
  std::vector<Point> out(d.size());
  for (u64 s = 0; s < d.size(); s++) out[s] = nat[natural_from_storage(d, s)];
  return out;
}

// Circle FFT twiddles (CircleCodeword.swift:129-171).
inline u64 fft_twiddle_offset(u32 stage, u64 n) { return stage == 0 ? 0 : n - (n >> stage); }
inline std::vector<u32> fft_twiddles(const Domain& d) {
  require(d.canonical() && d.storageOrder == 1);
  auto nat = natural_points(d);
  u64 n = d.size();
  std::vector<u32> tw;
  tw.reserve(n ? n - 1 : 0);
  for (u32 stage = 0; stage < d.logSize; stage++) {
    u64 cnt = n >> (stage + 1);
    for (u64 h = 0; h < cnt; h++) {
      Point p = nat[bit_reverse(h << (stage + 1), d.logSize)];
      if (stage == 0) { tw.push_back(p.y); continue; }
      u32 x = p.x;
      for (u32 k = 1; k < stage; k++) x = double_x(x);
      tw.push_back(x);
    }
  }
  return tw;
}

// Inverse-domain layers (CircleDomain.swift:399-418, 469-511, 545-562).  Returned as
// M31 values; the reference stores QM31(a: v, 0, 0, 0).
inline std::vector<std::vector<u32>> inverse_domain_layers(const Domain& d, u32 rounds) {
  require(d.storageOrder == 1 && d.canonical() && rounds > 0 && rounds <= d.logSize);
  auto nat = natural_points(d);
  u64 h = d.half();
  std::vector<u32> ys(h), xs(h);
  for (u64 i = 0; i < h; i++) {
    Point p = nat[bit_reverse(i << 1, d.logSize)];
    require(p.y != 0);
    ys[i] = p.y;
    xs[i] = p.x;
  }
  std::vector<std::vector<u32>> layers;
  std::vector<u32> inv(h);
  m31::batch_inverse(ys.data(), inv.data(), h);
  layers.push_back(inv);
  std::vector<u32> cur = xs;
  for (u32 r = 1; r < rounds; r++) {
    require(cur.size() > 1 && cur.size() % 2 == 0);
    u64 m = cur.size() / 2;
    std::vector<u32> left(m), nxt(m), li(m);
    for (u64 i = 0; i < m; i++) {
      u32 l = cur[2 * i], rr = cur[2 * i + 1];
      require(m31::add(l, rr) == 0 && l != 0);
      left[i] = l;
      nxt[i] = double_x(l);
    }
    m31::batch_inverse(left.data(), li.data(), m);
    layers.push_back(li);
    cur.swap(nxt);
  }
  return layers;
}

// ---------------------------------------------------------------------------
// Circle FFT codeword (CircleCodeword.swift:27-263)
// ---------------------------------------------------------------------------
struct Polynomial { std::vector<QM31> x, y; };

inline QM31 eval_univariate(const std::vector<QM31>& c, u32 x) {  // CircleCodeword.swift:173-185
  QM31 acc = {0, 0, 0, 0};
  for (size_t i = c.size(); i-- > 0;) acc = q_add(q_mul_m31(acc, x), c[i]);
  return acc;
}
inline QM31 eval_at(const Polynomial& p, Point pt) {  // CircleCodeword.swift:53-70
  validate_point(pt);
  return q_add(eval_univariate(p.x, pt.x), q_mul_m31(eval_univariate(p.y, pt.x), pt.y));
}
// Direct evaluation over the bit-reversed domain (CircleCodeword.swift:27-51).
inline std::vector<QM31> evaluate_direct(const Polynomial& p, const Domain& d) {
  require(d.canonical() && d.storageOrder == 1);
  auto nat = natural_points(d);
  std::vector<QM31> out(d.size());
#pragma omp parallel for schedule(static)
  for (long long s = 0; s < (long long)d.size(); s++) out[s] = eval_at(p, nat[bit_reverse(u64(s), d.logSize)]);
  return out;
}

inline std::vector<u32> cheb_mul_x(const std::vector<u32>& c) {  // CircleCodeword.swift:214-231
  static const u32 inv2 = 1073741824u;
  std::vector<u32> r(c.size() + 1, 0);
  for (size_t i = 0; i < c.size(); i++) {
    u32 v = c[i];
    if (!v) continue;
    if (i == 0) { r[1] = m31::add(r[1], v); continue; }
    u32 h = m31::mul(v, inv2);
    r[i - 1] = m31::add(r[i - 1], h);
    r[i + 1] = m31::add(r[i + 1], h);
  }
  return r;
}
inline std::vector<QM31> cheb_to_line(const std::vector<QM31>& c) {  // CircleCodeword.swift:233-263
  static const u32 inv2 = 1073741824u;
  require(!c.empty() && is_pow2(c.size()));
  if (c.size() == 1) return c;
  size_t half = c.size() / 2;
  std::vector<QM31> lo(c.begin(), c.begin() + half), hi(half, QM31{0, 0, 0, 0});
  hi[0] = c[half];
  if (half > 1) {
    for (size_t i = 1; i < half; i++) hi[i] = q_mul_m31(c[half + i], 2);
    for (size_t li = 1; li < half; li++) lo[li] = q_sub(lo[li], q_mul_m31(hi[half - li], inv2));
  }
  auto a = cheb_to_line(lo), b = cheb_to_line(hi);
  a.insert(a.end(), b.begin(), b.end());
  return a;
}
inline std::vector<QM31> line_basis(const std::vector<QM31>& mono, size_t capacity) {  // CircleCodeword.swift:187-212
  require(capacity > 0 && is_pow2(capacity) && mono.size() <= capacity);
  std::vector<QM31> ch(capacity, QM31{0, 0, 0, 0});
  if (mono.empty()) return ch;
  std::vector<u32> power = {1};
  for (size_t deg = 0; deg < mono.size(); deg++) {
    QM31 cf = mono[deg];
    if (!q_is_zero(cf))
      for (size_t i = 0; i < power.size(); i++)
        if (power[i]) ch[i] = q_add(ch[i], q_mul_m31(cf, power[i]));
    if (deg + 1 < mono.size()) power = cheb_mul_x(power);
  }
  return cheb_to_line(ch);
}
// Interleaved FFT-basis coefficients [x0,y0,x1,y1,...] (CircleCodeword.swift:100-127).
inline std::vector<QM31> fft_basis_coefficients(const Polynomial& p, const Domain& d) {
  require(d.canonical() && d.storageOrder == 1 && p.x.size() <= d.half() && p.y.size() <= d.half());
  auto xl = line_basis(p.x, d.half()), yl = line_basis(p.y, d.half());
  std::vector<QM31> out;
  out.reserve(d.size());
  for (u64 i = 0; i < d.half(); i++) { out.push_back(xl[i]); out.push_back(yl[i]); }
  return out;
}
// In-place butterflies, stages logN-1 ... 1 then 0 (CircleCodeword.swift:72-98).
inline void fft_in_place(std::vector<QM31>& v, const Domain& d, const std::vector<u32>& tw) {
  u64 n = d.size();
  require(v.size() == n && tw.size() == n - 1);
  std::vector<u32> stages;
  for (int s = int(d.logSize) - 1; s >= 1; s--) stages.push_back(u32(s));
  stages.push_back(0);
  for (u32 s : stages) {
    u64 cnt = n >> (s + 1), off = fft_twiddle_offset(s, n), span = u64(1) << s;
#pragma omp parallel for schedule(static)
    for (long long h = 0; h < (long long)cnt; h++) {
      u32 t = tw[off + h];
      for (u64 lane = 0; lane < span; lane++) {
        u64 l = (u64(h) << (s + 1)) + lane, r = l + span;
        QM31 sr = q_mul_m31(v[r], t), lv = v[l];
        v[l] = q_add(lv, sr);
        v[r] = q_sub(lv, sr);
      }
    }
  }
}
inline std::vector<QM31> evaluate_fft(const Polynomial& p, const Domain& d) {
  auto v = fft_basis_coefficients(p, d);
  fft_in_place(v, d, fft_twiddles(d));
  return v;
}

// ---------------------------------------------------------------------------
// FRI folding (QM31FRIFold.swift:11-44; CircleDomain.swift:446-465)
// ---------------------------------------------------------------------------
inline QM31 fold_pair(QM31 pos, QM31 neg, QM31 invPoint, QM31 ch) {
  QM31 even = q_add(pos, neg), odd = q_sub(pos, neg);
  QM31 oddAt = q_mul(odd, invPoint);
  QM31 mixed = q_add(even, q_mul(ch, oddAt));
  return q_mul(mixed, kInverseTwo);
}
inline std::vector<QM31> fold(const std::vector<QM31>& ev, const std::vector<QM31>& inv, QM31 ch) {
  require(ev.size() > 1 && ev.size() % 2 == 0 && inv.size() == ev.size() / 2);
  require(q_canonical(ch));
  for (auto& e : ev) require(q_canonical(e));
  for (auto& t : inv) require(q_canonical(t) && !q_is_zero(t));
  std::vector<QM31> out(ev.size() / 2);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < (long long)out.size(); i++) out[i] = fold_pair(ev[2 * i], ev[2 * i + 1], inv[i], ch);
  return out;
}
inline std::vector<QM31> lift(const std::vector<u32>& v) {
  std::vector<QM31> o(v.size());
  for (size_t i = 0; i < v.size(); i++) o[i] = {v[i], 0, 0, 0};
  return o;
}

// ---------------------------------------------------------------------------
// Merkle (MerkleOracle.swift:4-141), each tree built once and kept by level.
// levels[0] = leaf digests, levels.back() = {root}.
// ---------------------------------------------------------------------------
struct MerkleTree {
  std::vector<std::vector<Digest>> levels;
  const Digest& root() const { return levels.back()[0]; }
  size_t depth() const { return levels.size() - 1; }
  std::vector<Digest> siblings(u64 idx) const {
    std::vector<Digest> s;
    for (size_t l = 0; l + 1 < levels.size(); l++) { s.push_back(levels[l][idx ^ 1]); idx >>= 1; }
    return s;
  }
};
inline MerkleTree merkle_from_digests(std::vector<Digest> lvl) {
  require(!lvl.empty() && is_pow2(lvl.size()), Err::invalidLeafCount, "invalid leaf count", (long long)lvl.size());
  MerkleTree t;
  t.levels.push_back(std::move(lvl));
  while (t.levels.back().size() > 1) {
    const auto& cur = t.levels.back();
    std::vector<Digest> nxt(cur.size() / 2);
#pragma omp parallel for schedule(static) if (cur.size() > 4096)
    for (long long i = 0; i < (long long)nxt.size(); i++) nxt[i] = sha3_pair(cur[2 * i], cur[2 * i + 1]);
    t.levels.push_back(std::move(nxt));
  }
  return t;
}
inline MerkleTree merkle_raw(const u8* leaves, size_t nbytes, u64 count, u64 stride, u64 len) {
  require(count > 0 && is_pow2(count), Err::invalidLeafCount, "invalid leaf count", (long long)count);
  require(stride >= len);
  require(nbytes >= count * stride);
  std::vector<Digest> d(count);
#pragma omp parallel for schedule(static) if (count > 4096)
  for (long long i = 0; i < (long long)count; i++) d[i] = sha3_256(leaves + u64(i) * stride, len);
  return merkle_from_digests(std::move(d));
}
inline MerkleTree merkle_qm31(const std::vector<QM31>& layer) {
  Bytes b = pack_qm31(layer);
  return merkle_raw(b.data(), b.size(), layer.size(), 16, 16);
}
// Literal per-opening rebuild (MerkleOracle.swift:53-110).
inline std::vector<Digest> merkle_opening_literal(const u8* leaves, size_t nbytes, u64 count, u64 stride, u64 len, u64 index, Digest* root) {
  require(index < count);
  MerkleTree t = merkle_raw(leaves, nbytes, count, stride, len);
  if (root) *root = t.root();
  return t.siblings(index);
}
// MerkleOracle.swift:112-141
inline bool merkle_verify(const u8* leaf, size_t leafLen, u64 index, const std::vector<Digest>& sib, const Digest& root) {
  require(sib.size() < 63);
  require(index < (u64(1) << sib.size()));
  Digest cur = sha3_256(leaf, leafLen);
  for (size_t l = 0; l < sib.size(); l++) cur = ((index >> l) & 1) == 0 ? sha3_pair(cur, sib[l]) : sha3_pair(sib[l], cur);
  return cur == root;
}

// ---------------------------------------------------------------------------
// Circle FRI transcript V1 (CircleProofFormat.swift:684-983)
// ---------------------------------------------------------------------------
struct Security { u32 logBlowup = 0, queries = 0, foldingStep = 1, grindingBits = 0;
  u32 nominal() const { return logBlowup * queries + grindingBits; }
  bool operator==(const Security& o) const { return logBlowup == o.logBlowup && queries == o.queries && foldingStep == o.foldingStep && grindingBits == o.grindingBits; }
};
inline void validate_security(const Security& s) {  // CircleProofFormat.swift:129-158
  u64 bits = u64(s.logBlowup) * s.queries + s.grindingBits;
  require(s.logBlowup > 0 && s.queries > 0 && s.foldingStep > 0 && s.grindingBits <= 64 && bits <= 0xFFFFFFFFull);
}

namespace frame_v1 {
static const char* kDomain = "AppleZKProver.CircleFRI.PCS.V1";
inline Bytes base(u8 type) {  // :969-975
  Bytes f;
  put_u32(f, u32(std::strlen(kDomain)));
  put_str(f, kDomain);
  put_u32(f, 1);
  f.push_back(type);
  return f;
}
inline Bytes header() { Bytes f = base(0); put_u32(f, 1); put_u32(f, 1); put_u32(f, m31::P); put_u32(f, kGenerator.x); put_u32(f, kGenerator.y); return f; }
inline Bytes security(const Security& s) { Bytes f = base(1); put_u32(f, s.logBlowup); put_u32(f, s.queries); put_u32(f, s.foldingStep); put_u32(f, s.grindingBits); put_u32(f, s.nominal()); return f; }
inline Bytes public_input(u32 n) { Bytes f = base(2); put_u32(f, n); return f; }
inline Bytes commitment(u32 i, u32 n) { Bytes f = base(3); put_u32(f, i); put_u32(f, n); return f; }
inline Bytes challenge(u32 i) { Bytes f = base(4); put_u32(f, i); put_u32(f, m31::P); put_u32(f, 4); return f; }
inline Bytes final_layer(u64 cnt, u64 bytes) { Bytes f = base(5); put_u64(f, cnt); put_u64(f, bytes); return f; }
inline Bytes query(u32 q, u64 pairs) { Bytes f = base(6); put_u32(f, q); put_u64(f, pairs); return f; }
inline Bytes grinding(u32 bits, u32 nonceBytes) { Bytes f = base(7); put_u32(f, bits); put_u32(f, nonceBytes); return f; }
}  // namespace frame_v1

// CircleDomainDescriptorCodecV1.encode (CircleProofFormat.swift:71-93)
inline Bytes encode_domain(const Domain& d) {
  require(d.canonical());
  Bytes b = {0x41, 0x5a, 0x4b, 0x43, 0x44, 0x56, 0x31, 0x00};
  put_u32(b, 1); put_u32(b, m31::P); put_u32(b, kCircleLogOrder); put_u32(b, kGenerator.x); put_u32(b, kGenerator.y);
  put_u32(b, d.logSize); put_u32(b, d.halfCosetInitial); put_u32(b, d.halfCosetLogSize); put_u32(b, d.storageOrder);
  return b;
}
inline Domain decode_domain(const Bytes& b) {  // CircleProofFormat.swift:95-126
  require(b.size() == 44);
  static const u8 magic[8] = {0x41, 0x5a, 0x4b, 0x43, 0x44, 0x56, 0x31, 0x00};
  require(std::memcmp(b.data(), magic, 8) == 0);
  const u8* p = b.data() + 8;
  require(get_u32(p) == 1 && get_u32(p + 4) == m31::P && get_u32(p + 8) == kCircleLogOrder && get_u32(p + 12) == kGenerator.x && get_u32(p + 16) == kGenerator.y);
  Domain d;
  d.logSize = get_u32(p + 20);
  d.halfCosetInitial = get_u32(p + 24) & kCircleOrderMask;
  d.halfCosetLogSize = get_u32(p + 28);
  d.storageOrder = get_u32(p + 32);
  require(d.storageOrder <= 2);
  require(d.logSize >= 1 && d.logSize <= 30 && d.halfCosetLogSize <= 29 && d.halfCosetLogSize == d.logSize - 1);
  require(d.canonical());
  return d;
}

// Prefix state after the public-input digest (CircleProofFormat.swift:803-826).
inline Transcript transcript_prefix(const Domain& d, const Security& s, const Digest& pub) {
  Transcript t;
  t.absorb(frame_v1::header());
  t.absorb(encode_domain(d));
  t.absorb(frame_v1::security(s));
  t.absorb(frame_v1::public_input(32));
  t.absorb(pub);
  return t;
}
inline QM31 transcript_round(Transcript& t, u32 index, const Digest& commitment) {  // :819-826
  t.absorb(frame_v1::commitment(index, 32));
  t.absorb(commitment);
  t.absorb(frame_v1::challenge(index));
  auto l = t.squeeze_u32(4, m31::P);
  return {l[0], l[1], l[2], l[3]};
}
// deriveChallenges (CircleProofFormat.swift:723-740).
inline std::vector<QM31> derive_challenges(const Domain& d, const Security& s, const Digest& pub, const std::vector<Digest>& cm) {
  require(d.storageOrder == 1 && d.canonical() && !cm.empty());
  Transcript t = transcript_prefix(d, s, pub);
  std::vector<QM31> ch;
  for (u32 i = 0; i < cm.size(); i++) ch.push_back(transcript_round(t, i, cm[i]));
  return ch;
}
// digestMeetsTarget (CircleProofFormat.swift:662-681)
inline bool grinding_ok(const Bytes& digest, u32 bits) {
  if (bits > digest.size() * 8) return false;
  int rem = int(bits);
  size_t i = 0;
  while (rem >= 8) { if (digest[i]) return false; i++; rem -= 8; }
  if (rem == 0) return true;
  u8 mask = u8(0xff << (8 - rem));
  return (digest[i] & mask) == 0;
}
inline Bytes absorb_grinding(Transcript& t, u32 bits, u64 nonce) {  // :872-883
  t.absorb(frame_v1::grinding(bits, 8));
  Bytes nb;
  put_u64(nb, nonce);
  t.absorb(nb);
  return t.squeeze_bytes(32);
}
struct TranscriptResult { std::vector<QM31> challenges; std::vector<u32> queryPairs; };
inline Transcript transcript_after_final(const Domain& d, const Security& s, const Digest& pub, const std::vector<Digest>& cm,
                                         const std::vector<QM31>& finalLayer, std::vector<QM31>* ch) {  // :828-857
  require(d.storageOrder == 1 && d.canonical() && !cm.empty() && !finalLayer.empty());
  for (auto& v : finalLayer) require(q_canonical(v));
  Transcript t = transcript_prefix(d, s, pub);
  for (u32 i = 0; i < cm.size(); i++) { QM31 c = transcript_round(t, i, cm[i]); if (ch) ch->push_back(c); }
  Bytes fb = pack_qm31(finalLayer);
  t.absorb(frame_v1::final_layer(finalLayer.size(), fb.size()));
  t.absorb(fb);
  return t;
}
// findGrindingNonce (CircleProofFormat.swift:753-794)
inline bool find_grinding_nonce(const Domain& d, const Security& s, const Digest& pub, const std::vector<Digest>& cm,
                                const std::vector<QM31>& fl, u64* nonce) {
  if (s.grindingBits == 0) return false;
  require(s.grindingBits <= 20);
  Transcript base = transcript_after_final(d, s, pub, cm, fl, nullptr);
  for (u64 n = 0;; n++) {
    Transcript c = base;
    if (grinding_ok(absorb_grinding(c, s.grindingBits, n), s.grindingBits)) { *nonce = n; return true; }
  }
}
// derive (CircleProofFormat.swift:687-722)
inline TranscriptResult transcript_derive(const Domain& d, const Security& s, const Digest& pub, const std::vector<Digest>& cm,
                                          const std::vector<QM31>& fl, bool hasNonce, u64 nonce) {
  TranscriptResult r;
  Transcript t = transcript_after_final(d, s, pub, cm, fl, &r.challenges);
  if (s.grindingBits == 0) {
    require(!hasNonce);
  } else {
    require(hasNonce);
    require(grinding_ok(absorb_grinding(t, s.grindingBits, nonce), s.grindingBits));
  }
  t.absorb(frame_v1::query(s.queries, d.half()));
  r.queryPairs = t.squeeze_u32(s.queries, u32(d.half()));
  return r;
}

// ---------------------------------------------------------------------------
// Proof types + codec (CircleProofFormat.swift:288-645)
// ---------------------------------------------------------------------------
struct ValueOpening { u64 leafIndex = 0; QM31 value{}; std::vector<Digest> siblings; };
struct LayerOpening { u32 layerIndex = 0; u64 pairIndex = 0; ValueOpening left, right; };
struct Query { u64 initialPair = 0; std::vector<LayerOpening> layers; };
struct Proof {
  u32 version = 1, transcriptVersion = 1;
  Domain domain;
  Security security;
  Digest publicDigest{};
  std::vector<Digest> commitments;
  std::vector<QM31> finalLayer;
  std::vector<Query> queries;
  std::vector<ValueOpening> claimed;
  bool hasNonce = false;
  u64 nonce = 0;
};

inline void encode_opening(Bytes& d, const ValueOpening& o) {  // :582-593
  put_u64(d, o.leafIndex);
  put_qm31(d, o.value);
  put_u32(d, u32(o.siblings.size()));
  for (auto& s : o.siblings) d.insert(d.end(), s.b, s.b + 32);
}
inline Bytes encode_proof(const Proof& p) {  // :478-525
  Bytes d = {0x41, 0x5a, 0x4b, 0x50, 0x46, 0x56, 0x31, 0x00};
  put_u32(d, p.version);
  put_u32(d, p.transcriptVersion);
  Bytes db = encode_domain(p.domain);
  put_u32(d, u32(db.size()));
  put_bytes(d, db);
  put_u32(d, p.security.logBlowup); put_u32(d, p.security.queries); put_u32(d, p.security.foldingStep); put_u32(d, p.security.grindingBits);
  put_u32(d, 32);
  d.insert(d.end(), p.publicDigest.b, p.publicDigest.b + 32);
  put_u32(d, u32(p.commitments.size()));
  for (auto& c : p.commitments) d.insert(d.end(), c.b, c.b + 32);
  put_u64(d, p.finalLayer.size());
  for (auto& v : p.finalLayer) put_qm31(d, v);
  put_u32(d, u32(p.queries.size()));
  for (auto& q : p.queries) {
    put_u64(d, q.initialPair);
    put_u32(d, u32(q.layers.size()));
    for (auto& l : q.layers) { put_u32(d, l.layerIndex); put_u64(d, l.pairIndex); encode_opening(d, l.left); encode_opening(d, l.right); }
  }
  if (!p.claimed.empty() || p.hasNonce) {
    put_u32(d, u32(p.claimed.size()));
    for (auto& o : p.claimed) encode_opening(d, o);
  }
  if (p.hasNonce) put_u64(d, p.nonce);
  return d;
}

struct Reader {  // CanonicalByteReader, CircleProofFormat.swift:1790-1836
  const u8* p; size_t n, off = 0;
  Reader(const u8* p_, size_t n_) : p(p_), n(n_) {}
  bool at_end() const { return off == n; }
  const u8* take(size_t k) { require(k <= n - off); const u8* r = p + off; off += k; return r; }
  u32 u32_() { return get_u32(take(4)); }
  u64 u64_() { return get_u64(take(8)); }
  Bytes bytes(size_t k) { const u8* r = take(k); return Bytes(r, r + k); }
  void finish() const { require(off == n); }
};
inline ValueOpening decode_opening(Reader& r) {  // :595-614
  ValueOpening o;
  o.leafIndex = r.u64_();
  o.value = get_qm31(r.take(16));
  require(q_canonical(o.value));
  u32 sc = r.u32_();
  for (u32 i = 0; i < sc; i++) { Digest dg; std::memcpy(dg.b, r.take(32), 32); o.siblings.push_back(dg); }
  return o;
}
// Shape validation of CirclePCSFRIProofV1.init (CircleProofFormat.swift:346-460).
inline void validate_proof_shape(const Proof& p) {
  const Domain& d = p.domain;
  bool nonceShape = p.security.grindingBits > 0 ? p.hasNonce : !p.hasNonce;
  require(p.version == 1 && p.transcriptVersion == 1 && d.storageOrder == 1 && d.canonical() && p.security.foldingStep == 1 && nonceShape);
  require(!p.commitments.empty() && p.commitments.size() <= d.logSize);
  require(p.finalLayer.size() == (d.size() >> p.commitments.size()));
  require(p.queries.size() == p.security.queries);
  for (auto& v : p.finalLayer) require(q_canonical(v));
  for (auto& q : p.queries) {
    require(q.initialPair < d.half() && q.layers.size() == p.commitments.size() && !q.layers.empty());
    for (size_t ri = 0; ri < q.layers.size(); ri++) {
      auto& l = q.layers[ri];
      require(l.layerIndex == ri && l.pairIndex == (q.initialPair >> ri) && l.layerIndex < p.commitments.size() && l.layerIndex < d.logSize);
      u64 cnt = d.size() >> l.layerIndex;
      require(cnt > 1 && l.pairIndex < cnt / 2 && l.left.leafIndex == l.pairIndex * 2 && l.right.leafIndex == l.pairIndex * 2 + 1);
      require(l.left.siblings.size() == size_t(log2_floor(cnt)) && l.right.siblings.size() == size_t(log2_floor(cnt)));
    }
  }
  bool first = true;
  u64 prev = 0;
  for (auto& o : p.claimed) {
    require(o.leafIndex < d.size() && o.siblings.size() == size_t(log2_floor(d.size())) && (first || prev < o.leafIndex));
    first = false;
    prev = o.leafIndex;
  }
}
inline Proof decode_proof(const u8* b, size_t n) {  // :527-580
  Reader r(b, n);
  static const u8 magic[8] = {0x41, 0x5a, 0x4b, 0x50, 0x46, 0x56, 0x31, 0x00};
  require(std::memcmp(r.take(8), magic, 8) == 0);
  Proof p;
  p.version = r.u32_();
  p.transcriptVersion = r.u32_();
  u32 dl = r.u32_();
  p.domain = decode_domain(r.bytes(dl));
  p.security.logBlowup = r.u32_(); p.security.queries = r.u32_(); p.security.foldingStep = r.u32_(); p.security.grindingBits = r.u32_();
  validate_security(p.security);
  u32 pl = r.u32_();
  require(pl == 32);
  std::memcpy(p.publicDigest.b, r.take(32), 32);
  u32 cc = r.u32_();
  for (u32 i = 0; i < cc; i++) { Digest dg; std::memcpy(dg.b, r.take(32), 32); p.commitments.push_back(dg); }
  u64 fc = r.u64_();
  require(fc <= (n / 16));
  for (u64 i = 0; i < fc; i++) { QM31 v = get_qm31(r.take(16)); require(q_canonical(v)); p.finalLayer.push_back(v); }
  u32 qc = r.u32_();
  for (u32 qi = 0; qi < qc; qi++) {
    Query q;
    q.initialPair = r.u64_();
    u32 lc = r.u32_();
    for (u32 li = 0; li < lc; li++) {
      LayerOpening l;
      l.layerIndex = r.u32_();
      l.pairIndex = r.u64_();
      l.left = decode_opening(r);
      l.right = decode_opening(r);
      q.layers.push_back(std::move(l));
    }
    require(!q.layers.empty());
    p.queries.push_back(std::move(q));
  }
  if (!r.at_end()) {
    u32 oc = r.u32_();
    for (u32 i = 0; i < oc; i++) p.claimed.push_back(decode_opening(r));
    if (!r.at_end()) { p.hasNonce = true; p.nonce = r.u64_(); }
  }
  r.finish();
  validate_proof_shape(p);
  return p;
}

// ---------------------------------------------------------------------------
// Proof builder (CircleFRIProofBuilderV1.prove, CircleProofFormat.swift:1173-1285)
// ---------------------------------------------------------------------------
struct ProverTrace {  // everything the GPU path also produces, for parity tests
  std::vector<Digest> commitments;
  std::vector<QM31> challenges;
  std::vector<QM31> finalLayer;
  std::vector<u32> queryPairs;
};
inline Proof build_proof(const std::vector<QM31>& evaluations, const Domain& d, const Security& s, const Digest& pub,
                         u32 rounds, const std::vector<u64>& claimedIdx = {}, ProverTrace* trace = nullptr) {
  require(d.storageOrder == 1 && d.canonical() && evaluations.size() == d.size() && s.foldingStep == 1 && s.grindingBits <= 20 && rounds > 0 && rounds <= d.logSize);
  validate_security(s);
  for (auto& e : evaluations) require(q_canonical(e));
  std::vector<u64> claimed = claimedIdx;
  std::sort(claimed.begin(), claimed.end());
  for (size_t i = 0; i < claimed.size(); i++) require(claimed[i] < d.size() && (i == 0 || claimed[i - 1] < claimed[i]));

  auto inv = inverse_domain_layers(d, rounds);
  std::vector<std::vector<QM31>> layers;
  std::vector<MerkleTree> trees;
  std::vector<Digest> cm;
  std::vector<QM31> ch;
  Transcript t = transcript_prefix(d, s, pub);
  std::vector<QM31> cur = evaluations;
  for (u32 r = 0; r < rounds; r++) {
    layers.push_back(cur);
    trees.push_back(merkle_qm31(cur));
    cm.push_back(trees.back().root());
    QM31 c = transcript_round(t, r, cm.back());
    ch.push_back(c);
    cur = fold(cur, lift(inv[r]), c);
  }
  Proof p;
  p.domain = d;
  p.security = s;
  p.publicDigest = pub;
  p.commitments = cm;
  p.finalLayer = cur;
  p.hasNonce = find_grinding_nonce(d, s, pub, cm, cur, &p.nonce);
  TranscriptResult tr = transcript_derive(d, s, pub, cm, cur, p.hasNonce, p.nonce);
  if (!(tr.challenges.size() == ch.size() && std::equal(ch.begin(), ch.end(), tr.challenges.begin())))
    fail(Err::correctnessValidationFailed, "Circle FRI transcript challenge changed after final-layer binding.");
  for (u32 pair : tr.queryPairs) {  // makeQuery (:1287-1331)
    Query q;
    q.initialPair = pair;
    u64 cp = pair;
    for (u32 li = 0; li < layers.size(); li++) {
      require(cp < layers[li].size() / 2);
      LayerOpening lo;
      lo.layerIndex = li;
      lo.pairIndex = cp;
      lo.left = {cp * 2, layers[li][cp * 2], trees[li].siblings(cp * 2)};
      lo.right = {cp * 2 + 1, layers[li][cp * 2 + 1], trees[li].siblings(cp * 2 + 1)};
      q.layers.push_back(std::move(lo));
      cp >>= 1;
    }
    p.queries.push_back(std::move(q));
  }
  for (u64 idx : claimed) p.claimed.push_back({idx, evaluations[idx], trees[0].siblings(idx)});
  if (trace) { trace->commitments = cm; trace->challenges = ch; trace->finalLayer = cur; trace->queryPairs = tr.queryPairs; }
  validate_proof_shape(p);
  return p;
}

// The reference's builder as written (CircleProofFormat.swift:1173-1356): every
// round's challenge comes from deriveChallenges over all commitments so far (the
// transcript replayed from its prefix), and every query opening packs its layer
// and rebuilds that layer's whole Merkle tree (MerkleOracle.openingSHA3_256), so
// openings cost O(queries x rounds x N) permutations.  Same bytes as build_proof;
// the CPU baseline times it (on one thread) beside the efficient form.
inline Proof build_proof_literal(const std::vector<QM31>& evaluations, const Domain& d, const Security& s, const Digest& pub, u32 rounds) {
  require(d.storageOrder == 1 && d.canonical() && evaluations.size() == d.size() && s.foldingStep == 1 && s.grindingBits <= 20 && rounds > 0 && rounds <= d.logSize);
  validate_security(s);
  for (auto& e : evaluations) require(q_canonical(e));
  auto inv = inverse_domain_layers(d, rounds);
  std::vector<std::vector<QM31>> layers;
  std::vector<Digest> cm;
  std::vector<QM31> ch;
  std::vector<QM31> cur = evaluations;
  for (u32 r = 0; r < rounds; r++) {  // :1209-1242
    layers.push_back(cur);
    Bytes lb = pack_qm31(cur);
    cm.push_back(merkle_raw(lb.data(), lb.size(), cur.size(), 16, 16).root());
    std::vector<QM31> prefix = derive_challenges(d, s, pub, cm);
    require(prefix.size() == cm.size());
    ch.push_back(prefix[r]);
    cur = fold(cur, lift(inv[r]), prefix[r]);
  }
  Proof p;
  p.domain = d;
  p.security = s;
  p.publicDigest = pub;
  p.commitments = cm;
  p.finalLayer = cur;
  p.hasNonce = find_grinding_nonce(d, s, pub, cm, cur, &p.nonce);
  TranscriptResult tr = transcript_derive(d, s, pub, cm, cur, p.hasNonce, p.nonce);
  if (!(tr.challenges.size() == ch.size() && std::equal(ch.begin(), ch.end(), tr.challenges.begin())))
    fail(Err::correctnessValidationFailed, "Circle FRI transcript challenge changed after final-layer binding.");
  for (u32 pair : tr.queryPairs) {  // makeQuery / makeOpening (:1287-1356)
    Query q;
    q.initialPair = pair;
    u64 cp = pair;
    for (u32 li = 0; li < layers.size(); li++) {
      require(cp < layers[li].size() / 2);
      Bytes lb = pack_qm31(layers[li]);
      LayerOpening lo;
      lo.layerIndex = li;
      lo.pairIndex = cp;
      lo.left = {cp * 2, layers[li][cp * 2], merkle_opening_literal(lb.data(), lb.size(), layers[li].size(), 16, 16, cp * 2, nullptr)};
      lo.right = {cp * 2 + 1, layers[li][cp * 2 + 1], merkle_opening_literal(lb.data(), lb.size(), layers[li].size(), 16, 16, cp * 2 + 1, nullptr)};
      q.layers.push_back(std::move(lo));
      cp >>= 1;
    }
    p.queries.push_back(std::move(q));
  }
  validate_proof_shape(p);
  return p;
}

// ---------------------------------------------------------------------------
// Commit-and-fold chain with 64-byte Merkle leaves (4 consecutive QM31, little-
// endian, per leaf): the transcript frames and folds of build_proof (header,
// domain, security, public input, per round commitment + challenge), with each
// layer's root taken over n/4 leaves of 64 bytes (MerkleOracle.swift:4-51 on the
// packed layer).  The reference's verifier reads 16-byte leaves, so this chain has
// commitments, challenges and a final layer but no proof encoding.
// ---------------------------------------------------------------------------
inline ProverTrace commit_fold_chain_leaf64(const std::vector<QM31>& evaluations, const Domain& d, const Security& s, const Digest& pub, u32 rounds) {
  require(d.storageOrder == 1 && d.canonical() && evaluations.size() == d.size() && rounds > 0 && rounds + 1 <= d.logSize);
  validate_security(s);
  for (auto& e : evaluations) require(q_canonical(e));
  auto inv = inverse_domain_layers(d, rounds);
  ProverTrace tr;
  Transcript t = transcript_prefix(d, s, pub);
  std::vector<QM31> cur = evaluations;
  for (u32 r = 0; r < rounds; r++) {
    Bytes b = pack_qm31(cur);
    MerkleTree tree = merkle_raw(b.data(), b.size(), cur.size() / 4, 64, 64);
    tr.commitments.push_back(tree.root());
    QM31 c = transcript_round(t, r, tr.commitments.back());
    tr.challenges.push_back(c);
    cur = fold(cur, lift(inv[r]), c);
  }
  tr.finalLayer = cur;
  return tr;
}

// ---------------------------------------------------------------------------
// Verifier (CirclePCSFRIProofVerifierV1.verify, CircleProofFormat.swift:1397-1488)
// ---------------------------------------------------------------------------
inline bool verify_value_opening(const ValueOpening& o, const Digest& root, u64 idx, size_t sibCount) {
  if (o.leafIndex != idx || o.siblings.size() != sibCount) return false;
  Bytes leaf;
  put_qm31(leaf, o.value);
  return merkle_verify(leaf.data(), 16, idx, o.siblings, root);
}
inline bool verify_proof(const Proof& p, const Digest& pub) {
  const Domain& d = p.domain;
  if (!(p.publicDigest == pub) || p.security.foldingStep != 1 || p.commitments.empty() || p.commitments.size() > d.logSize ||
      p.finalLayer.size() != (d.size() >> p.commitments.size()))
    return false;
  TranscriptResult tr;
  try {
    tr = transcript_derive(d, p.security, p.publicDigest, p.commitments, p.finalLayer, p.hasNonce, p.nonce);
  } catch (const OracleError&) {
    return false;
  }
  if (tr.challenges.size() != p.commitments.size() || tr.queryPairs.size() != p.queries.size()) return false;
  auto inv = inverse_domain_layers(d, u32(p.commitments.size()));
  for (size_t qo = 0; qo < p.queries.size(); qo++) {
    u64 pair = tr.queryPairs[qo];
    const Query& q = p.queries[qo];
    if (q.initialPair != pair || q.layers.size() != p.commitments.size()) return false;
    bool haveExp = false;
    u64 expIdx = 0;
    QM31 expVal{};
    for (size_t r = 0; r < p.commitments.size(); r++) {
      const LayerOpening& l = q.layers[r];
      u64 cnt = d.size() >> r;
      if (l.layerIndex != r || l.pairIndex != pair || pair >= cnt / 2) return false;
      u64 li = pair * 2, ri = li + 1;
      size_t sc = size_t(log2_floor(cnt));
      if (!verify_value_opening(l.left, p.commitments[r], li, sc) || !verify_value_opening(l.right, p.commitments[r], ri, sc)) return false;
      if (haveExp) {
        if (expIdx == li) { if (expVal != l.left.value) return false; }
        else if (expIdx == ri) { if (expVal != l.right.value) return false; }
        else return false;
      }
      QM31 t = {inv[r][pair], 0, 0, 0};
      expVal = fold_pair(l.left.value, l.right.value, t, tr.challenges[r]);
      expIdx = pair;
      haveExp = true;
      pair >>= 1;
    }
    if (!haveExp || expIdx >= p.finalLayer.size() || p.finalLayer[expIdx] != expVal) return false;
  }
  return true;
}

// Polynomial-claim digest (CircleProofFormat.swift:1095-1151).
struct EvalClaim { u64 storageIndex; Point point; QM31 value; };
inline Digest polynomial_claim_digest(const Domain& d, const Polynomial& poly, const std::vector<EvalClaim>& claims) {
  static const char* kDom = "AppleZKProver.CirclePCS.PolynomialClaim.V1";
  auto base = [](u8 type) { Bytes f; put_u32(f, u32(std::strlen(kDom))); put_str(f, kDom); f.push_back(type); return f; };
  Bytes data;
  Bytes f0 = base(0);
  put_u32(f0, u32(std::strlen(kDom))); put_str(f0, kDom); put_u32(f0, 1); put_u32(f0, 1);
  put_bytes(data, f0);
  put_bytes(data, encode_domain(d));
  Bytes f1 = base(1);
  put_u32(f1, u32(poly.x.size())); put_u32(f1, u32(poly.y.size())); put_u32(f1, 16);
  put_bytes(data, f1);
  put_bytes(data, pack_qm31(poly.x));
  put_bytes(data, pack_qm31(poly.y));
  Bytes f2 = base(2);
  put_u32(f2, u32(claims.size()));
  put_bytes(data, f2);
  for (auto& c : claims) { put_u64(data, c.storageIndex); put_u32(data, c.point.x); put_u32(data, c.point.y); put_qm31(data, c.value); }
  return sha3_256(data);
}
// CirclePCSFRIPolynomialClaimV1.make (CircleProofFormat.swift:1044-1069).
inline std::vector<EvalClaim> make_claims(const Domain& d, const Polynomial& poly, std::vector<u64> idx) {
  require(!idx.empty());
  std::sort(idx.begin(), idx.end());
  std::vector<EvalClaim> c;
  for (size_t i = 0; i < idx.size(); i++) {
    require(idx[i] < d.size() && (i == 0 || idx[i - 1] < idx[i]));
    Point pt = domain_point(d, natural_from_storage(d, idx[i]));
    c.push_back({idx[i], pt, eval_at(poly, pt)});
  }
  return c;
}
// CirclePCSFRIContractVerifierV1.verify with a statement under a parameter set
// (CircleProofFormat.swift:1548-1611, 1658-1700, 1728-1752, 238-285).
inline bool verify_contract(const Proof& p, const Domain& d, const Polynomial& poly, const std::vector<u64>& claimIdx, const Security& profile) {
  // acceptsProofShape
  if (!(p.security == profile)) return false;
  if (!(d.storageOrder == 1 && d.canonical() && d.logSize > profile.logBlowup)) return false;
  if (p.commitments.size() != d.logSize - profile.logBlowup) return false;
  if (p.finalLayer.size() != (u64(1) << profile.logBlowup)) return false;
  for (auto& v : p.finalLayer) if (v != p.finalLayer[0]) return false;
  auto claims = make_claims(d, poly, claimIdx);
  if (p.claimed.size() != claims.size()) return false;
  // polynomial verifier
  Digest pub = polynomial_claim_digest(d, poly, claims);
  if (!(p.publicDigest == pub) || p.domain.logSize != d.logSize || p.domain.halfCosetInitial != d.halfCosetInitial) return false;
  u64 maxCoef = std::max<u64>(1, d.size() >> p.security.logBlowup);
  if (p.security.logBlowup > d.logSize || poly.x.size() > maxCoef || poly.y.size() > maxCoef) return false;
  if (!verify_proof(p, pub)) return false;
  for (size_t i = 0; i < claims.size(); i++) {
    const auto& c = claims[i];
    const auto& o = p.claimed[i];
    Point expect = domain_point(d, natural_from_storage(d, c.storageIndex));
    if (!(c.point == expect) || !(eval_at(poly, c.point) == c.value)) return false;
    if (o.leafIndex != c.storageIndex || o.value != c.value) return false;
    if (!verify_value_opening(o, p.commitments[0], c.storageIndex, size_t(log2_floor(d.size())))) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// QM31 FRI fold chain with its own framing (QM31FRIFold.swift:88-238, 769-862)
// ---------------------------------------------------------------------------
namespace frame_qm31 {
static const char* kDomain = "AppleZKProver.QM31FRI.FoldChain";
inline Bytes base(u8 type) { Bytes f; put_u32(f, u32(std::strlen(kDomain))); put_str(f, kDomain); put_u32(f, 1); f.push_back(type); return f; }
inline Bytes header(u64 inputCount, u32 rounds, u32 commitBytes) { Bytes f = base(0); put_u64(f, inputCount); put_u32(f, rounds); put_u32(f, m31::P); put_u32(f, 4); put_u32(f, commitBytes); return f; }
inline Bytes round(u32 r, u64 in, u64 out, u32 commitBytes) { Bytes f = base(1); put_u32(f, r); put_u64(f, in); put_u64(f, out); put_u32(f, commitBytes); return f; }
inline Bytes challenge(u32 r) { Bytes f = base(2); put_u32(f, r); put_u32(f, m31::P); put_u32(f, 4); return f; }
}  // namespace frame_qm31

inline std::vector<QM31> qm31_transcript_challenges(u64 inputCount, const std::vector<Digest>& commitments) {  // :91-125
  require(inputCount > 1 && !commitments.empty());
  Transcript t;
  t.absorb(frame_qm31::header(inputCount, u32(commitments.size()), 32));
  std::vector<QM31> ch;
  u64 cur = inputCount;
  for (u32 r = 0; r < commitments.size(); r++) {
    require(cur > 1 && cur % 2 == 0);
    t.absorb(frame_qm31::round(r, cur, cur / 2, 32));
    t.absorb(commitments[r]);
    t.absorb(frame_qm31::challenge(r));
    auto l = t.squeeze_u32(4, m31::P);
    ch.push_back({l[0], l[1], l[2], l[3]});
    cur /= 2;
  }
  return ch;
}
// QM31FRIMerkleFoldChainOracle.commitAndFold (QM31FRIFold.swift:164-238)
inline std::vector<QM31> qm31_merkle_fold_chain(const std::vector<QM31>& ev, const std::vector<std::vector<QM31>>& inv,
                                                std::vector<Digest>* cmOut, std::vector<QM31>* chOut) {
  require(!inv.empty() && ev.size() > 1 && is_pow2(ev.size()));
  Transcript t;
  t.absorb(frame_qm31::header(ev.size(), u32(inv.size()), 32));
  std::vector<QM31> cur = ev;
  for (u32 r = 0; r < inv.size(); r++) {
    require(inv[r].size() == cur.size() / 2);
    Digest root = merkle_qm31(cur).root();
    if (cmOut) cmOut->push_back(root);
    t.absorb(frame_qm31::round(r, cur.size(), cur.size() / 2, 32));
    t.absorb(root);
    t.absorb(frame_qm31::challenge(r));
    auto l = t.squeeze_u32(4, m31::P);
    QM31 c = {l[0], l[1], l[2], l[3]};
    if (chOut) chOut->push_back(c);
    cur = fold(cur, inv[r], c);
  }
  return cur;
}

// ---------------------------------------------------------------------------
// M31 sum-check (SumcheckOracle.swift:212-303 chunk; :797-1064 multilinear)
// ---------------------------------------------------------------------------
namespace frame_sc {
inline Bytes base(const char* dom, u8 type) { Bytes f; put_u32(f, u32(std::strlen(dom))); put_str(f, dom); put_u32(f, 1); f.push_back(type); return f; }
}
struct ChunkResult { std::vector<u32> finalVector, coefficients, challenges; };
inline ChunkResult sumcheck_chunk(const std::vector<u32>& ev, u32 rounds) {  // :213-272
  require(ev.size() > 1 && is_pow2(ev.size()) && rounds > 0 && rounds <= u32(log2_floor(ev.size())));
  for (u32 v : ev) require(v < m31::P);
  static const char* dom = "AppleZKProver.SumcheckChunk";
  Transcript t;
  Bytes h = frame_sc::base(dom, 0); put_u64(h, ev.size()); put_u32(h, rounds); put_u32(h, m31::P);
  t.absorb(h);
  ChunkResult res;
  std::vector<u32> cur = ev;
  for (u32 r = 0; r < rounds; r++) {
    size_t pc = cur.size() / 2;
    Bytes rf = frame_sc::base(dom, 1); put_u32(rf, r); put_u64(rf, cur.size()); put_u64(rf, pc * 2);
    t.absorb(rf);
    Bytes words;
    for (size_t i = 0; i < pc * 2; i++) put_u32(words, cur[i]);
    t.absorb(words);
    Bytes cf = frame_sc::base(dom, 2); put_u32(cf, r); put_u32(cf, m31::P);
    t.absorb(cf);
    u32 c = t.squeeze_u32(1, m31::P)[0];
    res.challenges.push_back(c);
    res.coefficients.insert(res.coefficients.end(), cur.begin(), cur.begin() + pc * 2);
    std::vector<u32> nx(pc);
    for (size_t i = 0; i < pc; i++) nx[i] = m31::add(cur[2 * i], m31::mul(cur[2 * i + 1], c));
    cur.swap(nx);
  }
  res.finalVector = cur;
  return res;
}
inline Digest sumcheck_digest_words(const std::vector<u32>& w) {  // :1288-1299
  static const char* dom = "AppleZKProver.M31Sumcheck.Words.V1";
  Bytes f; put_u32(f, u32(std::strlen(dom))); put_str(f, dom); put_u32(f, 1); put_u64(f, w.size());
  for (u32 v : w) put_u32(f, v);
  return sha3_256(f);
}
struct MultilinearProof {
  u64 laneCount = 0; u32 rounds = 0; u32 claimedSum = 0; Digest initialDigest{};
  std::vector<u32> r0, r1, challenges;
  u32 finalEvaluation = 0;
};
inline MultilinearProof sumcheck_multilinear(const std::vector<u32>& ev) {  // :797-868
  require(ev.size() > 1 && is_pow2(ev.size()));
  for (u32 v : ev) require(v < m31::P);
  static const char* dom = "AppleZKProver.M31MultilinearSumcheck";
  MultilinearProof p;
  p.laneCount = ev.size();
  p.rounds = u32(log2_floor(ev.size()));
  u32 sum = 0;
  for (u32 v : ev) sum = m31::add(sum, v);
  p.claimedSum = sum;
  p.initialDigest = sumcheck_digest_words(ev);
  Transcript t;
  Bytes h = frame_sc::base(dom, 0); put_u64(h, p.laneCount); put_u32(h, p.rounds); put_u32(h, p.claimedSum);
  h.insert(h.end(), p.initialDigest.b, p.initialDigest.b + 32);
  t.absorb(h);
  std::vector<u32> cur = ev;
  for (u32 r = 0; r < p.rounds; r++) {
    u32 z = 0, o = 0;
    for (size_t i = 0; i < cur.size() / 2; i++) { z = m31::add(z, cur[2 * i]); o = m31::add(o, cur[2 * i + 1]); }
    p.r0.push_back(z);
    p.r1.push_back(o);
    Bytes rf = frame_sc::base(dom, 1); put_u32(rf, r); put_u32(rf, z); put_u32(rf, o);
    t.absorb(rf);
    Bytes cf = frame_sc::base(dom, 2); put_u32(cf, r); put_u32(cf, m31::P);
    t.absorb(cf);
    u32 c = t.squeeze_u32(1, m31::P)[0];
    p.challenges.push_back(c);
    u32 omc = m31::sub(1, c);
    std::vector<u32> nx(cur.size() / 2);
    for (size_t i = 0; i < nx.size(); i++) nx[i] = m31::add(m31::mul(omc, cur[2 * i]), m31::mul(c, cur[2 * i + 1]));
    cur.swap(nx);
  }
  require(cur.size() == 1);
  p.finalEvaluation = cur[0];
  return p;
}

}  // namespace azk_oracle
