"""Extract the reference's own golden vectors into tests/golden/ fixtures.

Run where a checkout of the reference is available, naming its root either as the
first argument or in AZK_REFERENCE_ROOT:

    python tests/golden/make_golden.py <reference root>

It reads the reference's XCTest sources, its checked-in benchmark JSON reports and
its proof corpus, and writes:

  reference_vectors.json   every known answer, with the reference file:line it came from
  corpus_valid.bin         CirclePCSFRIProofCorpusV1 valid proof bytes
  corpus_developer.bin     the corpus' "developer-parameter" proof bytes
  (the two single-byte tamper vectors are stored as (offset, byte) patches)

The tests never read the reference tree; they read only these fixtures.
"""
from __future__ import annotations

import json
import os
import re
import sys

ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("AZK_REFERENCE_ROOT", "")
HERE = os.path.dirname(os.path.abspath(__file__))
TESTS = "Tests/AppleZKProverTests"
BENCH = "BenchmarkBaselines"


def read(rel):
    with open(os.path.join(ROOT, rel), encoding="utf-8") as f:
        return f.read()


def line_of(text, needle, start=0):
    idx = text.index(needle, start)
    return text.count("\n", 0, idx) + 1, idx


def hex_after(text, needle, count=1):
    """The first `count` 64-hex-digit literals after `needle`."""
    line, idx = line_of(text, needle)
    found = re.findall(r'"([0-9a-f]{64})"', text[idx:])
    return line, found[:count]


def main():
    out = {"source": "reference tests and benchmark baselines", "vectors": {}}
    V = out["vectors"]

    sha = f"{TESTS}/SHA3OracleTests.swift"
    t = read(sha)
    ln, (h,) = hex_after(t, "func testEmptyStringVector")
    V["sha3_empty"] = {"hex": h, "ref": f"{sha}:{ln}"}
    ln, (h,) = hex_after(t, "func testABCStringVector")
    V["sha3_abc"] = {"hex": h, "ref": f"{sha}:{ln}"}
    ln, (h,) = hex_after(t, "func testKeccakEmptyStringVector")
    V["keccak_empty"] = {"hex": h, "ref": f"{sha}:{ln}"}
    ln, (h,) = hex_after(t, "func testKeccakABCStringVector")
    V["keccak_abc"] = {"hex": h, "ref": f"{sha}:{ln}"}
    for name, fn in (("sha3_rate_boundary", "func testSHA3RateBoundaryVectors"), ("keccak_rate_boundary", "func testKeccakRateBoundaryVectors")):
        ln, idx = line_of(t, fn)
        seg = t[idx: t.index("for (length", idx)]
        pairs = re.findall(r'\((\d+),\s*"([0-9a-f]{64})"\)', seg)
        V[name] = {"pattern": "byte i = (i*11 + 7) mod 256", "cases": [[int(a), b] for a, b in pairs], "ref": f"{sha}:{ln}"}

    mk = f"{TESTS}/MerkleTests.swift"
    t = read(mk)
    ln, (h,) = hex_after(t, "func testCPUDeterministicMerkleRoot")
    V["merkle_root_8x32"] = {"hex": h, "count": 8, "length": 32, "salt": 0, "generator": "byte(leaf,j) = leaf*29 + j*7 + salt + 3", "ref": f"{mk}:{ln}"}
    ln, (h,) = hex_after(t, "func testCPULargeRawMerkleRootMatchesDataLeaves")
    V["merkle_root_1024x32_salt71"] = {"hex": h, "count": 1024, "length": 32, "salt": 71, "ref": f"{mk}:{ln}"}

    pl = f"{TESTS}/PlannerTests.swift"
    t = read(pl)
    ln, idx = line_of(t, "func testTranscriptSqueezeUsesFullRateAndAdditionalBlocks")
    seg = t[idx: t.index("try transcript.absorb", idx)]
    words = [int(w.replace("_", "")) for w in re.findall(r"\b([0-9][0-9_]*)\b", seg.split("let expected")[1])]
    V["transcript_squeeze_40"] = {"input": "513 bytes, byte i = (i*31) mod 256", "words": words, "ref": f"{pl}:{ln}"}
    ln, idx = line_of(t, "func testM31SumcheckCPUOracleStableFramedTranscriptVector")
    seg = t[idx: t.index("func testTranscriptStateAbsorbsMultipleBlocks", idx)]

    def arr(after):
        s = seg.index(after)
        body = seg[seg.index("[", s) + 1: seg.index("]", s)]
        return [int(w.replace("_", "")) for w in re.findall(r"[0-9][0-9_]*", body)]

    V["sumcheck_chunk_16x3"] = {"input": "e[i] = (i+1)*17, 16 lanes, 3 rounds", "final": arr("result.finalVector"), "challenges": arr("result.challenges"),
                                "coefficients": arr("result.coefficients"), "ref": f"{pl}:{ln}"}

    cd = f"{TESTS}/CircleDomainTests.swift"
    t = read(cd)
    ln, hs = hex_after(t, "func testCircleDomainAndTwiddleStableVectorDigests", 3)
    V["circle_log5_digests"] = {"points": hs[0], "fft_twiddles": hs[1], "inverse_layers_4": hs[2], "ref": f"{cd}:{ln}"}
    ln, (h,) = hex_after(t, "func testCircleFirstFoldStableVectorDigest")
    V["circle_first_fold_proof_log4"] = {"hex": h, "log": 4, "security": [2, 3, 1, 0], "public": "0x10+i", "rounds": 1, "ref": f"{cd}:{ln}"}
    ln, (h,) = hex_after(t, "func testCircleMultiLayerFRIProofVerifierAndStableDigest")
    V["circle_3round_proof_log5"] = {"hex": h, "log": 5, "security": [2, 5, 1, 0], "public": "0x50+i", "rounds": 3, "ref": f"{cd}:{ln}"}
    ln, _ = line_of(t, "func testCircleDomainIndexAndLayoutPolicyMatchesCanonicalOrder")
    V["circle_layout_log3"] = {"natural_indices_over_2^27": [1, 5, 9, 13, 15, 11, 7, 3], "circle_to_coset": [0, 2, 4, 6, 7, 5, 3, 1],
                               "coset_to_circle": [0, 7, 1, 6, 2, 5, 3, 4], "ref": f"{cd}:{ln}"}
    # verify those literals are present verbatim
    for lit in ("1, 5, 9, 13, 15, 11, 7, 3", "[0, 2, 4, 6, 7, 5, 3, 1]", "[0, 7, 1, 6, 2, 5, 3, 4]"):
        assert lit in t, lit

    # benchmark baselines (log-14 / log-10 digests)
    def bench(fn, *path):
        d = json.loads(read(f"{BENCH}/{fn}"))
        for p in path:
            d = d[p]
        return d

    V["bench_circle_first_fold_log14"] = {"hex": bench("apple-m4-circle-fri-fold-2026-04-13.json", "verification", "cpuOutputDigestHex"),
                                          "salts": [0xC31, 0xC37, 0xC3D, 0xC43], "challenge": [41, 43, 47, 53],
                                          "ref": f"{BENCH}/apple-m4-circle-fri-fold-2026-04-13.json"}
    V["bench_circle_fold_chain_explicit_log14"] = {"hex": bench("apple-m4-circle-fri-fold-chain-2026-04-14.json", "verification", "cpuOutputDigestHex"),
                                                   "salts": [0xCC1, 0xCC7, 0xCCD, 0xCD3], "rounds": 3,
                                                   "ref": f"{BENCH}/apple-m4-circle-fri-fold-chain-2026-04-14.json"}
    V["bench_circle_fold_chain_merkle_log14"] = {"hex": bench("apple-m4-circle-fri-fold-chain-merkle-2026-04-14.json", "verification", "cpuOutputDigestHex"),
                                                 "salts": [0xCC1, 0xCC7, 0xCCD, 0xCD3], "rounds": 3, "security": [2, 4, 1, 0], "public": "0x90+i",
                                                 "proof_bytes": bench("apple-m4-circle-fri-fold-chain-merkle-2026-04-14.json", "proofSizeBytes"),
                                                 "ref": f"{BENCH}/apple-m4-circle-fri-fold-chain-merkle-2026-04-14.json"}
    for log, fn in ((14, "apple-m4-circle-codeword-prover-2026-04-14.json"), (10, "apple-m4-circle-codeword-fft-prover-2026-04-14.json")):
        V[f"bench_codeword_prover_log{log}"] = {"codeword_hex": bench(fn, "verification", "cpuCodewordDigestHex"),
                                                "proof_hex": bench(fn, "verification", "cpuProofDigestHex"),
                                                "proof_bytes": bench(fn, "proofSizeBytes"), "rounds": 3, "queries": 4, "security": [2, 4, 1, 0],
                                                "public": "0xa0+i", "x_salts": [0xE01, 0xE03, 0xE07, 0xE0B], "y_salts": [0xE11, 0xE17, 0xE1D, 0xE23],
                                                "x_count": 8, "y_count": 7, "ref": f"{BENCH}/{fn}"}
    suite = json.loads(read(f"{BENCH}/apple-m4-apple9-suite-2026-04-13.json"))
    roots = {}
    for rep in suite["reports"]:
        roots[str(rep["configuration"]["leafLength"])] = rep["verification"]["cpuRootHex"]
    V["bench_merkle_roots_16384"] = {"roots_by_leaf_length": roots, "generator": "byte(leaf,j) = leaf*131 + j*17 + 0x5a, stride = length",
                                     "ref": f"{BENCH}/apple-m4-apple9-suite-2026-04-13.json"}

    # proof corpus
    corpus_rel = f"{TESTS}/Resources/CirclePCSFRIProofCorpusV1.json"
    c = json.loads(read(corpus_rel))
    valid = bytes.fromhex(c["validCase"]["proofHex"])
    with open(os.path.join(HERE, "corpus_valid.bin"), "wb") as f:
        f.write(valid)
    tampers = []
    for tv in c["tamperVectors"]:
        b = bytes.fromhex(tv["proofHex"])
        entry = {"id": tv["id"], "expected_accepted": tv["expectedVerifierAccepted"], "bytes": tv["proofByteCount"], "digest": tv["proofDigestHex"]}
        if len(b) == len(valid) and sum(1 for i in range(len(b)) if b[i] != valid[i]) <= 4:
            entry["patch"] = [[i, b[i]] for i in range(len(b)) if b[i] != valid[i]]
        else:
            fname = "corpus_developer.bin"
            with open(os.path.join(HERE, fname), "wb") as f:
                f.write(b)
            entry["file"] = fname
        tampers.append(entry)
    vc = c["validCase"]
    V["corpus"] = {"profile": c["profile"], "log": vc["domainLogSize"], "rounds": vc["roundCount"], "claimed": vc["claimedStorageIndices"],
                   "x_hex": vc["xCoefficientHex"], "y_hex": vc["yCoefficientHex"], "public_digest": vc["publicInputDigestHex"],
                   "valid_digest": vc["proofDigestHex"], "valid_bytes": vc["proofByteCount"], "valid_file": "corpus_valid.bin",
                   "tampers": tampers, "ref": corpus_rel}

    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", len(V), "vector groups")


if __name__ == "__main__":
    if not ROOT:
        sys.exit("usage: make_golden.py <reference root> (or set AZK_REFERENCE_ROOT)")
    if not os.path.isdir(ROOT):
        sys.exit(f"reference checkout not found at {ROOT}")
    main()
