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
import ctypes
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
    if "fold" in which:
        # QM31 fold of 2^log values with QM31 inverse points: 16n read + 8n inverse
        # read + 8n write bytes (n inputs), one launch

        ev = np.zeros((n, 4), np.uint32)
        ev[:] = rng.integers(0, 2**31 - 1, size=ev.shape, dtype=np.uint32)
        inv = rng.integers(1, 2**31 - 1, size=(n // 2, 4), dtype=np.uint32)
        ch = np.array([[11, 13, 17, 19]], np.uint32)
        res = np.empty((n // 2, 4), np.uint32)
        ts = []
        for _ in range(reps + 1):
            st = azk.Stats()
            azk._capi.check(azk.lib().azk_qm31_fold(ctx.handle, ev.ctypes.data, n, inv.ctypes.data, ch.ctypes.data, res.ctypes.data, ctypes.byref(st)),
                            ctx.handle)
            ts.append(st.gpu_s)
        t = statistics.median(ts[1:])
        hbm, kind = _hbm_peak()
        emit({"what": "qm31 fold (QM31 inverse points)", "count": n, "seconds": t, "hbm_gbs": 32 * n / t / 1e9, "frac_hbm": 32 * n / t / 1e9 / hbm,
              "peak_source": kind})
        # Circle fold of one layer with M31 inverse twiddles: 16n read + 2n twiddle
        # read + 8n write bytes (n inputs), as in the superstep's final folds
        ts = []
        chs = np.array([[11, 13, 17, 19]], np.uint32)
        for _ in range(reps + 1):
            st = azk.Stats()
            azk._capi.check(azk.lib().azk_circle_fold_chain(ctx.handle, log_count, ev.ctypes.data, chs.ctypes.data, 1, res.ctypes.data,
                                                            ctypes.byref(st)), ctx.handle)
            ts.append(st.gpu_s)
        t = statistics.median(ts[1:])
        emit({"what": "circle fold, one layer (M31 inverse twiddles)", "count": n, "seconds": t, "hbm_gbs": 26 * n / t / 1e9,
              "frac_hbm": 26 * n / t / 1e9 / hbm, "peak_source": kind})
    if "fft" in which:
        # Circle FFT stage of a batch of 16 log-22 instances (blowup 4): lifted M31
        # coefficients (one-limb path) and full QM31 coefficients
        lg, cnt = 22, 16
        rows = (1 << lg) >> 2
        for label, limbs in (("lifted M31", 1), ("QM31", 4)):
            flat = np.zeros((rows * cnt, 4), np.uint32)
            flat[:, :limbs] = rng.integers(0, 2**31 - 1, size=(rows * cnt, limbs), dtype=np.uint32)
            b = azk.BatchProver(ctx, [lg] * cnt, [lg - 6] * cnt, 2, 64)
            b.upload(flat, [rows * i for i in range(cnt)], [rows] * cnt)
            pubs = bytes(32 * cnt)
            b.prove(pubs)
            b.set_profiling(True)
            fs = []
            for _ in range(reps):
                b.prove(pubs)
                fs.append(b.profile()["fft_s"])
            t = statistics.median(fs)
            N = (1 << lg) * cnt
            alg = 16 * N + 16 * N + 4 * N
            hbm, kind = _hbm_peak()
            emit({"what": f"circle fft 16 x log 22, {label} coefficients", "seconds": t, "elems_per_s": N / t, "hbm_gbs": alg / t / 1e9,
                  "frac_hbm": alg / t / 1e9 / hbm, "algorithmic": "16N read + 16N write + 4N twiddles", "peak_source": kind})
            del b
    if "sumcheck" in which:
        # M31 multilinear sum-check over 2^20 evaluations: the statement digest (one
        # sequential SHA3 sponge over the 4 MiB table, 30,841 permutations) and the
        # 20 rounds, device time of the two kernels
        ev = rng.integers(0, 2**31 - 1, size=1 << 20, dtype=np.uint32)
        ts = []
        for _ in range(reps + 1):
            st = azk.Stats()
            r0, r1, ch = (np.zeros(20, np.uint32) for _ in range(3))
            cs, fe, dg = ctypes.c_uint32(), ctypes.c_uint32(), np.zeros(32, np.uint8)
            azk._capi.check(azk.lib().azk_sumcheck_prove(ctx.handle, ev.ctypes.data, len(ev), r0.ctypes.data, r1.ctypes.data, ch.ctypes.data,
                                                         ctypes.byref(cs), ctypes.byref(fe), dg.ctypes.data, ctypes.byref(st)), ctx.handle)
            ts.append(st.gpu_s)
        t = statistics.median(ts[1:])
        perms = (50 + 4 * len(ev)) // 136 + 1
        emit({"what": "m31 multilinear sum-check 2^20 (digest + 20 rounds)", "seconds": t, "digest_permutations": perms,
              "us_per_permutation": t / perms * 1e6})
    ctx.close()
    return out


def _hbm_peak():
    import json
    import os

    try:
        with open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", default="perm,sha3,merkle,prove,fold,fft,sumcheck")
    ap.add_argument("--log", type=int, default=24)
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    run(a.which.split(","), a.log, a.reps)


if __name__ == "__main__":
    main()
