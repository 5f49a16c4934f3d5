// Device-side sponge transcript and the Circle FRI V1 frames.
//
// absorb() pads and permutes on every call; squeeze_u32() works on a copy of the
// state, 34 little-endian u32 words per block, rejection-sampling candidates at
// or above 2^32 - (2^32 mod m) (SHA3Oracle.swift:8-98; the reference's GPU twin is
// HashMerkleKernels.metal:1324-1404).  Frames are byte-identical to
// CircleFRITranscriptV1 (CircleProofFormat.swift:906-975) and
// QM31FRIFoldTranscriptFraming (QM31FRIFold.swift:769-862).
//
// Transcript work is a handful of permutations per round, run by one thread.
#pragma once
#include <stdint.h>
#include "azk_keccak.cuh"

namespace azk {

struct Transcript {
  uint64_t st[25];
};

__host__ __device__ inline void tr_reset(Transcript& t) {
  for (int i = 0; i < 25; i++) t.st[i] = 0;
}

__host__ __device__ inline void tr_permute(uint64_t (&s)[25]) { keccak_f1600<1>(s); }

// XOR byte k of a block into the state.
__host__ __device__ inline void tr_xor_byte(uint64_t (&s)[25], int k, uint8_t v) { s[k >> 3] ^= (uint64_t)v << (8 * (k & 7)); }

// Absorb `len` bytes from p (any address space readable by the caller).
__host__ __device__ inline void tr_absorb(Transcript& t, const uint8_t* p, uint32_t len, uint8_t suffix = 0x06) {
  uint32_t off = 0;
  while (off + 136 <= len) {
    for (int k = 0; k < 136; k++) tr_xor_byte(t.st, k, p[off + k]);
    tr_permute(t.st);
    off += 136;
  }
  uint32_t tail = len - off;
  for (uint32_t k = 0; k < tail; k++) tr_xor_byte(t.st, (int)k, p[off + k]);
  tr_xor_byte(t.st, (int)tail, suffix);
  tr_xor_byte(t.st, 135, 0x80);
  tr_permute(t.st);
}

// Absorb a 32-byte digest given as four little-endian lanes.
__host__ __device__ inline void tr_absorb_digest(Transcript& t, const uint64_t (&d)[4]) {
  for (int i = 0; i < 4; i++) t.st[i] ^= d[i];
  t.st[4] ^= 0x06;
  t.st[16] ^= kPadEnd;
  tr_permute(t.st);
}

// Squeeze `count` words mod `modulus` from a copy of the state.
__host__ __device__ inline void tr_squeeze_u32(const Transcript& t, uint32_t count, uint32_t modulus, uint32_t* out) {
  uint64_t s[25];
  for (int i = 0; i < 25; i++) s[i] = t.st[i];
  const uint64_t space = 1ull << 32;
  const uint64_t limit = space - (space % modulus);
  uint32_t produced = 0, idx = 0;
  while (produced < count) {
    if (idx > 0 && idx % 34 == 0) tr_permute(s);
    uint32_t w = idx % 34;
    uint64_t cand = (uint32_t)(s[w >> 1] >> ((w & 1) * 32));
    idx++;
    if (cand < limit) out[produced++] = (uint32_t)(cand % modulus);
  }
}

// First `count` (<= 136) squeeze bytes from a copy of the state.
__host__ __device__ inline void tr_squeeze_bytes(const Transcript& t, uint32_t count, uint8_t* out) {
  for (uint32_t b = 0; b < count; b++) out[b] = (uint8_t)(t.st[b >> 3] >> (8 * (b & 7)));
}

// ---- frame builders (little-endian) ----
struct FrameBuf {
  uint8_t b[136];
  uint32_t n;
};
__host__ __device__ inline void fb_u8(FrameBuf& f, uint8_t v) { f.b[f.n++] = v; }
__host__ __device__ inline void fb_u32(FrameBuf& f, uint32_t v) {
  for (int i = 0; i < 4; i++) f.b[f.n++] = (uint8_t)(v >> (8 * i));
}
__host__ __device__ inline void fb_u64(FrameBuf& f, uint64_t v) {
  for (int i = 0; i < 8; i++) f.b[f.n++] = (uint8_t)(v >> (8 * i));
}
__host__ __device__ inline void fb_str(FrameBuf& f, const char* s, uint32_t n) {
  for (uint32_t i = 0; i < n; i++) f.b[f.n++] = (uint8_t)s[i];
}

// Circle FRI PCS V1 base frame: u32 len || "AppleZKProver.CircleFRI.PCS.V1" || u32 1 || u8 type
__host__ __device__ inline void circle_frame(FrameBuf& f, uint8_t type) {
  const char dom[] = "AppleZKProver.CircleFRI.PCS.V1";
  f.n = 0;
  fb_u32(f, 30);
  fb_str(f, dom, 30);
  fb_u32(f, 1);
  fb_u8(f, type);
}
// QM31 fold-chain base frame: u32 len || "AppleZKProver.QM31FRI.FoldChain" || u32 1 || u8 type
__host__ __device__ inline void qm31_frame(FrameBuf& f, uint8_t type) {
  const char dom[] = "AppleZKProver.QM31FRI.FoldChain";
  f.n = 0;
  fb_u32(f, 31);
  fb_str(f, dom, 31);
  fb_u32(f, 1);
  fb_u8(f, type);
}

// Circle V1 round: commitment frame, root, challenge frame, squeeze 4 limbs.
__host__ __device__ inline void circle_round(Transcript& t, uint32_t round, const uint64_t (&root)[4], uint32_t (&ch)[4]) {
  FrameBuf f;
  circle_frame(f, 3);
  fb_u32(f, round);
  fb_u32(f, 32);
  tr_absorb(t, f.b, f.n);
  tr_absorb_digest(t, root);
  circle_frame(f, 4);
  fb_u32(f, round);
  fb_u32(f, 2147483647u);
  fb_u32(f, 4);
  tr_absorb(t, f.b, f.n);
  tr_squeeze_u32(t, 4, 2147483647u, ch);
}

// QM31 fold-chain round (QM31FRIFold.swift:203-213).
__host__ __device__ inline void qm31_round(Transcript& t, uint32_t round, uint64_t inCount, const uint64_t (&root)[4], uint32_t (&ch)[4]) {
  FrameBuf f;
  qm31_frame(f, 1);
  fb_u32(f, round);
  fb_u64(f, inCount);
  fb_u64(f, inCount / 2);
  fb_u32(f, 32);
  tr_absorb(t, f.b, f.n);
  tr_absorb_digest(t, root);
  qm31_frame(f, 2);
  fb_u32(f, round);
  fb_u32(f, 2147483647u);
  fb_u32(f, 4);
  tr_absorb(t, f.b, f.n);
  tr_squeeze_u32(t, 4, 2147483647u, ch);
}

}  // namespace azk
