// C-ABI over the CPU oracle (azk_oracle.hpp) for the Python tests, smoke() and the
// bench's CPU baseline.  CPU ORACLE: test infrastructure, never linked into the
// CUDA library.
//
// Every function returns 0 on success or a positive AppleZKProverError-like code
// (see azk_oracle::Err); azko_last_error() holds the message of the last failure.
#include "azk_oracle.hpp"

using namespace azk_oracle;

static thread_local std::string g_err;

#define AZKO_TRY try {
#define AZKO_CATCH                                                   \
  }                                                                  \
  catch (const OracleError& e) { g_err = e.what(); return int(e.kind); } \
  catch (const std::exception& e) { g_err = e.what(); return 99; }    \
  return 0;

static std::vector<QM31> q_vec(const u32* p, u64 n) {
  std::vector<QM31> v(n);
  for (u64 i = 0; i < n; i++) v[i] = {p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]};
  return v;
}
static void q_out(const std::vector<QM31>& v, u32* p) {
  for (size_t i = 0; i < v.size(); i++) { p[4 * i] = v[i].a; p[4 * i + 1] = v[i].b; p[4 * i + 2] = v[i].c; p[4 * i + 3] = v[i].d; }
}
static Digest dg(const u8* p) { Digest d; std::memcpy(d.b, p, 32); return d; }

extern "C" {

const char* azko_last_error() { return g_err.c_str(); }

int azko_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void azko_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Keccak-f[1600] over `count` states at byte stride `stride` (in place).
int azko_keccak_f1600(u8* states, u64 count, u64 stride) {
  AZKO_TRY
  require(stride >= 200 && stride % 8 == 0);
#pragma omp parallel for schedule(static) if (count > 1024)
  for (long long i = 0; i < (long long)count; i++) {
    u64 s[25];
    std::memcpy(s, states + u64(i) * stride, 200);
    keccak_f1600(s);
    std::memcpy(states + u64(i) * stride, s, 200);
  }
  AZKO_CATCH
}

int azko_sha3_256(const u8* data, u64 n, u8* out) { AZKO_TRY Digest d = sha3_256(data, n); std::memcpy(out, d.b, 32); AZKO_CATCH }
int azko_keccak_256(const u8* data, u64 n, u8* out) { AZKO_TRY Digest d = keccak_256(data, n); std::memcpy(out, d.b, 32); AZKO_CATCH }

// Fixed-length batch hashing; output padding bytes beyond 32 are zeroed like the
// reference plans (SHA3BatchHasher.swift:175-177).
int azko_hash_batch(const u8* msgs, u64 count, u64 stride, u64 len, u8* out, u64 outStride, int keccak) {
  AZKO_TRY
  require(len <= 136, Err::unsupportedOneBlockLength, "unsupported one-block length", (long long)len);
  require(count > 0 && stride >= len && outStride >= 32);
#pragma omp parallel for schedule(static) if (count > 1024)
  for (long long i = 0; i < (long long)count; i++) {
    Digest d = keccak ? keccak_256(msgs + u64(i) * stride, len) : sha3_256(msgs + u64(i) * stride, len);
    u8* o = out + u64(i) * outStride;
    std::memcpy(o, d.b, 32);
    if (outStride > 32) std::memset(o + 32, 0, outStride - 32);
  }
  AZKO_CATCH
}

int azko_merkle_root(const u8* leaves, u64 nbytes, u64 count, u64 stride, u64 len, u8* root) {
  AZKO_TRY
  require(len <= 136, Err::unsupportedOneBlockLength, "unsupported one-block length", (long long)len);
  MerkleTree t = merkle_raw(leaves, nbytes, count, stride, len);
  std::memcpy(root, t.root().b, 32);
  AZKO_CATCH
}

// Openings for several leaves of one tree (tree built once); siblings_out holds
// indexCount * depth digests, bottom-up per leaf.
int azko_merkle_openings(const u8* leaves, u64 nbytes, u64 count, u64 stride, u64 len, const u64* idx, u64 nidx,
                         u8* siblings_out, u8* root) {
  AZKO_TRY
  MerkleTree t = merkle_raw(leaves, nbytes, count, stride, len);
  size_t depth = t.depth();
  for (u64 k = 0; k < nidx; k++) {
    require(idx[k] < count);
    auto s = t.siblings(idx[k]);
    for (size_t l = 0; l < depth; l++) std::memcpy(siblings_out + (k * depth + l) * 32, s[l].b, 32);
  }
  std::memcpy(root, t.root().b, 32);
  AZKO_CATCH
}

// The reference's literal opening: full tree rebuild for one leaf (MerkleOracle.swift:53-110).
int azko_merkle_opening_literal(const u8* leaves, u64 nbytes, u64 count, u64 stride, u64 len, u64 index, u8* siblings_out, u8* root) {
  AZKO_TRY
  Digest r;
  auto s = merkle_opening_literal(leaves, nbytes, count, stride, len, index, &r);
  for (size_t l = 0; l < s.size(); l++) std::memcpy(siblings_out + l * 32, s[l].b, 32);
  std::memcpy(root, r.b, 32);
  AZKO_CATCH
}

// returns 1 valid, 0 invalid, negative on malformed input
int azko_merkle_verify(const u8* leaf, u64 leafLen, u64 index, const u8* siblings, u64 depth, const u8* root) {
  try {
    std::vector<Digest> s(depth);
    for (u64 l = 0; l < depth; l++) s[l] = dg(siblings + 32 * l);
    return merkle_verify(leaf, leafLen, index, s, dg(root)) ? 1 : 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

int azko_merkle_root_prehashed(const u8* digests, u64 count, u8* root) {
  AZKO_TRY
  std::vector<Digest> d(count);
  for (u64 i = 0; i < count; i++) d[i] = dg(digests + 32 * i);
  MerkleTree t = merkle_from_digests(std::move(d));
  std::memcpy(root, t.root().b, 32);
  AZKO_CATCH
}

// All tree levels of a QM31 layer (16-byte leaves) concatenated: level 0 first.
int azko_merkle_qm31_levels(const u32* layer, u64 n, u8* levels_out) {
  AZKO_TRY
  MerkleTree t = merkle_qm31(q_vec(layer, n));
  size_t off = 0;
  for (auto& lvl : t.levels) for (auto& d : lvl) { std::memcpy(levels_out + off, d.b, 32); off += 32; }
  AZKO_CATCH
}

// Transcript: absorb each of `nframes` frames, then squeeze `count` words mod `modulus`.
int azko_transcript_squeeze(const u8* data, const u64* frameLens, u64 nframes, u64 count, u32 modulus, u32* out) {
  AZKO_TRY
  Transcript t;
  u64 off = 0;
  for (u64 f = 0; f < nframes; f++) { t.absorb(data + off, frameLens[f]); off += frameLens[f]; }
  auto w = t.squeeze_u32(count, modulus);
  std::memcpy(out, w.data(), 4 * w.size());
  AZKO_CATCH
}

int azko_transcript_state(const u8* data, const u64* frameLens, u64 nframes, u64* state_out) {
  AZKO_TRY
  Transcript t;
  u64 off = 0;
  for (u64 f = 0; f < nframes; f++) { t.absorb(data + off, frameLens[f]); off += frameLens[f]; }
  std::memcpy(state_out, t.st, 200);
  AZKO_CATCH
}

int azko_qm31_mul(const u32* x, const u32* y, u32* out) {
  AZKO_TRY QM31 r = q_mul({x[0], x[1], x[2], x[3]}, {y[0], y[1], y[2], y[3]}); q_out({r}, out); AZKO_CATCH
}
int azko_qm31_inv(const u32* x, u32* out) { AZKO_TRY QM31 r = q_inv({x[0], x[1], x[2], x[3]}); q_out({r}, out); AZKO_CATCH }

// Domain points in storage (bit-reversed) order as (x, y) pairs.
int azko_domain_points(u32 logSize, u32* xy) {
  AZKO_TRY
  Domain d = canonical_domain(logSize);
  auto p = storage_points(d);
  for (size_t i = 0; i < p.size(); i++) { xy[2 * i] = p[i].x; xy[2 * i + 1] = p[i].y; }
  AZKO_CATCH
}
int azko_domain_encode(u32 logSize, u8* out44) { AZKO_TRY Bytes b = encode_domain(canonical_domain(logSize)); std::memcpy(out44, b.data(), 44); AZKO_CATCH }

int azko_fft_twiddles(u32 logSize, u32* out) {
  AZKO_TRY
  auto t = fft_twiddles(canonical_domain(logSize));
  std::memcpy(out, t.data(), 4 * t.size());
  AZKO_CATCH
}
// Concatenated inverse-domain layers as M31 words: N/2 + N/4 + ... (rounds layers).
int azko_inverse_layers(u32 logSize, u32 rounds, u32* out) {
  AZKO_TRY
  auto L = inverse_domain_layers(canonical_domain(logSize), rounds);
  size_t off = 0;
  for (auto& l : L) { std::memcpy(out + off, l.data(), 4 * l.size()); off += l.size(); }
  AZKO_CATCH
}

int azko_fft_basis_coefficients(u32 logSize, const u32* x, u64 nx, const u32* y, u64 ny, u32* out) {
  AZKO_TRY
  Polynomial p{q_vec(x, nx), q_vec(y, ny)};
  q_out(fft_basis_coefficients(p, canonical_domain(logSize)), out);
  AZKO_CATCH
}
int azko_evaluate_direct(u32 logSize, const u32* x, u64 nx, const u32* y, u64 ny, u32* out) {
  AZKO_TRY
  Polynomial p{q_vec(x, nx), q_vec(y, ny)};
  q_out(evaluate_direct(p, canonical_domain(logSize)), out);
  AZKO_CATCH
}
// In-place FFT of N interleaved FFT-basis coefficients into the bit-reversed codeword.
int azko_fft_evaluate(u32 logSize, u32* values) {
  AZKO_TRY
  Domain d = canonical_domain(logSize);
  auto v = q_vec(values, d.size());
  fft_in_place(v, d, fft_twiddles(d));
  q_out(v, values);
  AZKO_CATCH
}

// One QM31 fold with an explicit QM31 inverse-domain layer.
int azko_fold(const u32* ev, u64 n, const u32* inv, const u32* ch, u32* out) {
  AZKO_TRY
  q_out(fold(q_vec(ev, n), q_vec(inv, n / 2), {ch[0], ch[1], ch[2], ch[3]}), out);
  AZKO_CATCH
}
// Circle fold chain with explicit challenges (CircleFRILayerOracleV1.fold, CircleDomain.swift:513-543).
int azko_circle_fold_chain(u32 logSize, const u32* ev, const u32* ch, u32 rounds, u32* out) {
  AZKO_TRY
  Domain d = canonical_domain(logSize);
  auto inv = inverse_domain_layers(d, rounds);
  auto cur = q_vec(ev, d.size());
  for (u32 r = 0; r < rounds; r++) cur = fold(cur, lift(inv[r]), {ch[4 * r], ch[4 * r + 1], ch[4 * r + 2], ch[4 * r + 3]});
  q_out(cur, out);
  AZKO_CATCH
}

// QM31 FRI transcript-derived challenges (QM31FRIFoldTranscriptOracle.deriveChallenges).
int azko_qm31_transcript_challenges(u64 inputCount, const u8* commitments, u32 rounds, u32* out) {
  AZKO_TRY
  std::vector<Digest> c(rounds);
  for (u32 r = 0; r < rounds; r++) c[r] = dg(commitments + 32 * r);
  q_out(qm31_transcript_challenges(inputCount, c), out);
  AZKO_CATCH
}
// QM31FRIMerkleFoldChainOracle.commitAndFold with explicit QM31 inverse layers (concatenated).
int azko_qm31_merkle_fold_chain(const u32* ev, u64 n, const u32* invLayers, u32 rounds, u32* finalOut, u8* commitOut, u32* chOut) {
  AZKO_TRY
  std::vector<std::vector<QM31>> inv;
  u64 off = 0, cnt = n / 2;
  for (u32 r = 0; r < rounds; r++) { inv.push_back(q_vec(invLayers + 4 * off, cnt)); off += cnt; cnt /= 2; }
  std::vector<Digest> cm;
  std::vector<QM31> ch;
  auto f = qm31_merkle_fold_chain(q_vec(ev, n), inv, &cm, &ch);
  q_out(f, finalOut);
  for (u32 r = 0; r < rounds; r++) std::memcpy(commitOut + 32 * r, cm[r].b, 32);
  q_out(ch, chOut);
  AZKO_CATCH
}

// Circle PCS/FRI proof (CircleFRIProofBuilderV1.prove).  Writes the encoded proof
// (proofLen in/out: capacity in, size out) and the trace the GPU path also emits.
int azko_prove(u32 logSize, const u32* evaluations, u32 logBlowup, u32 queries, u32 grindingBits, const u8* pub, u32 rounds,
               const u64* claimed, u64 nclaimed, u8* proofOut, u64* proofLen, u8* commitOut, u32* chOut, u32* finalOut,
               u32* queryPairsOut) {
  AZKO_TRY
  Domain d = canonical_domain(logSize);
  Security s{logBlowup, queries, 1, grindingBits};
  ProverTrace tr;
  std::vector<u64> cl(claimed, claimed + nclaimed);
  Proof p = build_proof(q_vec(evaluations, d.size()), d, s, dg(pub), rounds, cl, &tr);
  Bytes b = encode_proof(p);
  require(b.size() <= *proofLen, Err::invalidInputLayout, "proof buffer too small");
  std::memcpy(proofOut, b.data(), b.size());
  *proofLen = b.size();
  if (commitOut) for (u32 r = 0; r < rounds; r++) std::memcpy(commitOut + 32 * r, tr.commitments[r].b, 32);
  if (chOut) q_out(tr.challenges, chOut);
  if (finalOut) q_out(tr.finalLayer, finalOut);
  if (queryPairsOut) std::memcpy(queryPairsOut, tr.queryPairs.data(), 4 * tr.queryPairs.size());
  AZKO_CATCH
}

// The reference's literal single-thread form from FFT-basis coefficients: the
// stage-by-stage FFT (CircleCodeword.swift:72-98) and build_proof_literal, with the
// oracle's thread count held at one for the call.
int azko_prove_literal(u32 logSize, const u32* coefficients, u32 logBlowup, u32 queries, const u8* pub, u32 rounds, u8* proofOut, u64* proofLen) {
#ifdef _OPENMP
  const int saved = omp_get_max_threads();
  omp_set_num_threads(1);
#endif
  int rc = 0;
  try {
    Domain d = canonical_domain(logSize);
    Security s{logBlowup, queries, 1, 0};
    auto v = q_vec(coefficients, d.size());
    fft_in_place(v, d, fft_twiddles(d));
    Bytes b = encode_proof(build_proof_literal(v, d, s, dg(pub), rounds));
    require(b.size() <= *proofLen, Err::invalidInputLayout, "proof buffer too small");
    std::memcpy(proofOut, b.data(), b.size());
    *proofLen = b.size();
  } catch (const OracleError& e) {
    g_err = e.what();
    rc = int(e.kind);
  } catch (const std::exception& e) {
    g_err = e.what();
    rc = 99;
  }
#ifdef _OPENMP
  omp_set_num_threads(saved);
#endif
  return rc;
}

int azko_commit_fold_chain_leaf64(u32 logSize, const u32* evaluations, u32 logBlowup, u32 queries, const u8* pub, u32 rounds, u8* commitOut,
                                  u32* chOut, u32* finalOut) {
  AZKO_TRY
  Domain d = canonical_domain(logSize);
  Security s{logBlowup, queries, 1, 0};
  ProverTrace tr = commit_fold_chain_leaf64(q_vec(evaluations, d.size()), d, s, dg(pub), rounds);
  for (u32 r = 0; r < rounds; r++) std::memcpy(commitOut + 32 * r, tr.commitments[r].b, 32);
  q_out(tr.challenges, chOut);
  q_out(tr.finalLayer, finalOut);
  AZKO_CATCH
}

// 1 accepted, 0 rejected, negative if the bytes do not decode.
int azko_verify(const u8* proof, u64 n, const u8* pub) {
  try {
    Proof p = decode_proof(proof, n);
    return verify_proof(p, dg(pub)) ? 1 : 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
// Decode then re-encode; returns 0 when the round trip is byte-identical.
int azko_proof_roundtrip(const u8* proof, u64 n) {
  AZKO_TRY
  Proof p = decode_proof(proof, n);
  Bytes b = encode_proof(p);
  require(b.size() == n && std::memcmp(b.data(), proof, n) == 0, Err::correctnessValidationFailed, "round trip mismatch");
  AZKO_CATCH
}
int azko_verify_contract(const u8* proof, u64 n, u32 logSize, const u32* x, u64 nx, const u32* y, u64 ny, const u64* idx, u64 nidx,
                         u32 logBlowup, u32 queries, u32 grindingBits) {
  try {
    Proof p = decode_proof(proof, n);
    Polynomial poly{q_vec(x, nx), q_vec(y, ny)};
    std::vector<u64> ix(idx, idx + nidx);
    return verify_contract(p, canonical_domain(logSize), poly, ix, Security{logBlowup, queries, 1, grindingBits}) ? 1 : 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}
int azko_claim_digest(u32 logSize, const u32* x, u64 nx, const u32* y, u64 ny, const u64* idx, u64 nidx, u8* out) {
  AZKO_TRY
  Domain d = canonical_domain(logSize);
  Polynomial poly{q_vec(x, nx), q_vec(y, ny)};
  auto claims = make_claims(d, poly, std::vector<u64>(idx, idx + nidx));
  Digest g = polynomial_claim_digest(d, poly, claims);
  std::memcpy(out, g.b, 32);
  AZKO_CATCH
}

int azko_sumcheck_chunk(const u32* ev, u64 n, u32 rounds, u32* finalOut, u32* coeffOut, u32* chOut) {
  AZKO_TRY
  auto r = sumcheck_chunk(std::vector<u32>(ev, ev + n), rounds);
  std::memcpy(finalOut, r.finalVector.data(), 4 * r.finalVector.size());
  std::memcpy(coeffOut, r.coefficients.data(), 4 * r.coefficients.size());
  std::memcpy(chOut, r.challenges.data(), 4 * r.challenges.size());
  AZKO_CATCH
}
// Multilinear sum-check: r0/r1/challenges have log2(n) words; returns claimed sum,
// final evaluation and the initial-evaluation digest.
int azko_sumcheck_multilinear(const u32* ev, u64 n, u32* r0, u32* r1, u32* ch, u32* claimedSum, u32* finalEval, u8* initialDigest) {
  AZKO_TRY
  auto p = sumcheck_multilinear(std::vector<u32>(ev, ev + n));
  std::memcpy(r0, p.r0.data(), 4 * p.rounds);
  std::memcpy(r1, p.r1.data(), 4 * p.rounds);
  std::memcpy(ch, p.challenges.data(), 4 * p.rounds);
  *claimedSum = p.claimedSum;
  *finalEval = p.finalEvaluation;
  std::memcpy(initialDigest, p.initialDigest.b, 32);
  AZKO_CATCH
}

}  // extern "C"
