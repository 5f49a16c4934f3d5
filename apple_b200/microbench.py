"""Primitive throughput on one B200 (the survey's C2 and C3 configurations).

    python -m apple_b200.microbench [--which perm,sha3,merkle,prove] [--log 24]

Prints one JSON line per measurement.  Inputs are seeded random bytes / M31 values
resident in device memory; every kernel time is CUDA-event device time over
repeated launches after warm-up (inputs of 2^24 items are larger than the 126 MB
L2).  Keccak rates are compared with the device's measured LOP3+SHF issue rate
(azk_probe_int_issue / 4320 ops per permutation).
"""
from __future__ import annotations

import argparse
import json
import statistics

import numpy as np

import apple_b200 as azk


def _rand_bytes(rng, n):
    return rng.integers(0, 256, size=n, dtype=np.uint8)


def run(which, log_count, reps=5):
    ctx = azk.Context(0)
    rng = np.random.default_rng(0xA11CE002)
    peak = azk.probe_int_issue(ctx) / 4320.0
    n = 1 << log_count
    out = []

    def emit(d):
        d.setdefault("perm_peak_per_s", peak)
        if "perms_per_s" in d:
            d["frac_int_roofline"] = d["perms_per_s"] / peak
        print(json.dumps(d), flush=True)
        out.append(d)

    if "perm" in which:
        buf = ctx.alloc(200 * n)
        buf.upload(_rand_bytes(rng, 200 * n))
        res = ctx.alloc(200 * n)
        plan = azk.KeccakF1600PermutationPlan(ctx, n)
        for _ in range(2):
            plan.permute_resident(buf.ptr, res.ptr)
        t = statistics.median(plan.permute_resident(buf.ptr, res.ptr).gpu_s for _ in range(reps))
        emit({"what": "keccak-f1600 batch", "count": n, "seconds": t, "perms_per_s": n / t, "hbm_gbs": 400 * n / t / 1e9})
        del buf, res
    if "sha3" in which:
        for length in (32, 64, 128, 136):
            buf = ctx.alloc(length * n)
            buf.upload(_rand_bytes(rng, length * n))
            res = ctx.alloc(32 * n)
            plan = azk.SHA3FixedOneBlockHashPlan(ctx, n, length, length)
            for _ in range(2):
                plan.hash_resident(buf.ptr, res.ptr)
            t = statistics.median(plan.hash_resident(buf.ptr, res.ptr).gpu_s for _ in range(reps))
            perms = n * (2 if length == 136 else 1)
            emit({"what": f"sha3-256 batch {length} B", "count": n, "seconds": t, "hashes_per_s": n / t, "perms_per_s": perms / t})
            del buf, res
    if "merkle" in which:
        buf = ctx.alloc(64 * n)
        buf.upload(_rand_bytes(rng, 64 * n))
        for tl in (9, 10, 11, 12, 13):
            plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, n, 64, 64, treelet_log=tl)
            plan.commit_resident(buf.ptr)
            ts = []
            for _ in range(reps):
                plan.commit_resident(buf.ptr)
                ts.append(plan.last_stats.gpu_s)
            t = statistics.median(ts)
            idx = rng.integers(0, n, size=1024)
            paths = plan.open_resident(idx)
            ot = plan.last_stats.cpu_wall_s
            emit({"what": "sha3 merkle commit 64 B leaves", "treelet_log": tl, "count": n, "seconds": t, "perms_per_s": (2 * n - 1) / t,
                  "openings": len(paths), "openings_wall_s": ot})
            plan.close()
        del buf
    if "prove" in which:
        lg = 22
        coeffs = np.zeros(((1 << lg) // 4, 4), np.uint32)
        coeffs[:, 0] = rng.integers(0, 2**31 - 1, size=len(coeffs), dtype=np.uint32)
        pub = bytes(range(32))
        prover = azk.CirclePCSFRIProver(ctx, lg, 2, 64, 16, schedule=dict(treelet_log=12, group_log=12))
        prover.prove_coefficients(coeffs, pub)
        ts = []
        for _ in range(reps):
            prover.prove_coefficients(coeffs, pub)
            ts.append(prover.last_stats.gpu_s)
        t = statistics.median(ts)
        perms = sum(2 * ((1 << lg) >> k) - 1 + 3 for k in range(16))
        emit({"what": "circle pcs prove log 22 (FFT + 16 rounds + 64 queries + proof bytes), single instance", "seconds": t,
              "elems_per_s": (1 << lg) / t, "perms_per_s": perms / t, "wall_s": prover.last_stats.cpu_wall_s})
    ctx.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", default="perm,sha3,merkle,prove")
    ap.add_argument("--log", type=int, default=24)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    run(a.which.split(","), a.log, a.reps)


if __name__ == "__main__":
    main()
