"""Benchmark: batched commit-and-fold superstep on B200 (one JSON line).

Workload (default): 512 independent Circle PCS/FRI commit-and-fold instances with
log codeword sizes drawn uniformly in [10, 22] (SplitMix64 seed 0xA11CE004),
blowup 4 (the low quarter of each interleaved FFT-basis coefficient buffer holds
seeded uniform M31 values lifted to QM31, the rest is zero), 16-byte QM31 Merkle
leaves, SHA3 Merkle commitment per layer, QM31 Circle FRI folds down to log 6
with Merkle-transcript challenges, 64 queries, proof bytes emitted on device.

Metric: committed-and-folded codeword elements per second (sum of 2^logN over
the instances / device time of one superstep).  `e2e` is the same metric through
the C ABI from pinned host buffers: coefficients H2D, prove, proof bytes D2H.
`plain` is the per-instance form (each instance's kernels launched in sequence).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one replica per GPU (torchrun; instances do not exchange data, so
there is no collective on the data path) and reports the max device time over
ranks.  `--impl reference` times the CPU restatement of the reference's CPU
oracle on the host cores instead (the reference itself is Swift + Metal and cannot
run on this box).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

# one hardware work queue per stream (the provers, server workers and copies run
# on many streams); read when CUDA initialises, so set before torch starts it
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 0xA11CE004
P = 2147483647


def splitmix64(seed, n):
    GOLD = np.uint64(0x9E3779B97F4A7C15)
    k = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + k * GOLD
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_m31(seed, n):
    out, draw = [], 0
    have = 0
    while have < n:
        w = splitmix64((seed + 0x51ED27 * draw) & 0xFFFFFFFFFFFFFFFF, n - have + (n - have) // 16 + 16)
        v = (w & np.uint64(0x7FFFFFFF)).astype(np.uint32)
        v = v[v != np.uint32(P)]
        out.append(v)
        have += len(v)
        draw += 1
    return np.concatenate(out)[:n]


def workload(count=512, lo=10, hi=22, final_log=6, seed=SEED):
    """Log sizes, rounds and the compact coefficient prefix of every instance."""
    draws = splitmix64(seed, count)
    logs = [int(lo + (int(d) % (hi - lo + 1))) for d in draws]
    rounds = [max(1, lg - final_log) for lg in logs]
    counts = [(1 << lg) >> 2 for lg in logs]  # blowup 4: the low quarter carries the coefficients
    offsets = list(np.cumsum([0] + counts[:-1]))
    return logs, rounds, counts, offsets


def coefficient_rows(counts, seed=SEED):
    total = int(sum(counts))
    rows = np.zeros((total, 4), np.uint32)
    rows[:, 0] = uniform_m31(seed ^ 0xC0EFF, total)
    return rows


def public_digests(n, seed=SEED):
    w = splitmix64(seed ^ 0x9B, 4 * n)
    return w.astype("<u8").tobytes()


class ClockSampler:
    """nvidia-smi clocks/throttle reasons during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower() == "active":
                    reasons.add(name)
        loaded = [v for v in sm if smax and v > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def tuned_tables():
    """The tuned per-layer treelet tables the library was built with (apple_b200/tuned_b200.json)."""
    try:
        with open(os.path.join(ROOT, "apple_b200", "tuned_b200.json")) as f:
            return {k: {int(lg): int(t) for lg, t in v.items()} for k, v in json.load(f)["tables"].items()}
    except (OSError, ValueError, KeyError):
        return None


def tuned_thread_tables():
    """The tuned per-layer thread counts the library was built with, if any."""
    try:
        with open(os.path.join(ROOT, "apple_b200", "tuned_b200.json")) as f:
            return {k: {int(lg): int(t) for lg, t in v.items()} for k, v in json.load(f).get("thread_tables", {}).items()}
    except (OSError, ValueError, KeyError):
        return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d.get("hbm_gbs"), "measured"
    except (OSError, ValueError):
        return 6650.0, "fallback"


def profile_traffic():
    """dram bytes per launch of the tree kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def dist_backend() -> str:
    """NCCL on GPU boxes; gloo where no CUDA device exists (the CPU tests of the
    multi-rank path), or whatever AZK_DIST_BACKEND names."""
    import torch

    return os.environ.get("AZK_DIST_BACKEND") or ("nccl" if torch.cuda.is_available() else "gloo")


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = dist_backend()
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, value: float, local: int) -> float:
    if dist is None:
        return value
    import torch

    device = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def stratified_sample(logs, max_log=64):
    """One instance of each log size present up to `max_log` (the first of each,
    smallest size first).  The workload draws log sizes uniformly, so the full
    sample has the workload's size mix."""
    first = {}
    for i, lg in enumerate(logs):
        if lg <= max_log:
            first.setdefault(lg, i)
    return [first[lg] for lg in sorted(first)]


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_sample(logs, rounds, counts, offsets, rows, pubs, sample):
    """Prove the instances `sample` with the CPU oracle (all host threads): FFT of the
    coefficients, then the proof.  Returns (elements, seconds, proofs)."""
    from oracle import pyoracle as O

    t0 = time.perf_counter()
    elems = 0
    proofs = {}
    for i in sample:
        lg = logs[i]
        n = 1 << lg
        c = np.zeros((n, 4), np.uint32)
        c[: counts[i]] = rows[offsets[i]:offsets[i] + counts[i]]
        ev = O.fft_evaluate(lg, c)
        proofs[i] = O.prove(lg, ev, 2, 64, pubs[32 * i:32 * i + 32], rounds[i]).proof
        elems += n
    dt = time.perf_counter() - t0
    return elems, dt, proofs


def cpu_literal_sample(logs, rounds, counts, offsets, rows, pubs, max_log=14):
    """The reference's literal single-thread builder (a full layer re-hash per opening,
    CircleProofFormat.swift:1287-1356) on the sampled instances of log size <=
    `max_log`, one host thread.  Returns (elements, seconds, proofs)."""
    from oracle import pyoracle as O

    sample = [i for i in stratified_sample(logs) if logs[i] <= max_log]
    t0 = time.perf_counter()
    elems = 0
    proofs = {}
    for i in sample:
        lg = logs[i]
        n = 1 << lg
        c = np.zeros((n, 4), np.uint32)
        c[: counts[i]] = rows[offsets[i]:offsets[i] + counts[i]]
        proofs[i] = O.prove_literal(lg, c, 2, 64, pubs[32 * i:32 * i + 32], rounds[i])
        elems += n
    return elems, time.perf_counter() - t0, proofs


def verify_all(proofs, pubs):
    """The oracle's verifier over every proof, on all host threads."""
    import concurrent.futures as cf

    from oracle import pyoracle as O

    def one(i):
        return O.verify(proofs[i], pubs[32 * i:32 * i + 32])

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        return list(ex.map(one, range(len(proofs))))


def run_reference(args, logs, rounds, counts, offsets, rows, pubs, world, rank, dist):
    if rank != 0:
        return
    from oracle import pyoracle as O

    O.lib()
    threads = O.num_threads()
    sample = stratified_sample(logs, args.cpu_max_log)
    small = [i for i in sample if logs[i] <= 12]
    for _ in range(args.warmup):
        cpu_sample(logs, rounds, counts, offsets, rows, pubs, small[:2])
    total_t, total_e = 0.0, 0
    for _ in range(args.steps):
        e, dt, _ = cpu_sample(logs, rounds, counts, offsets, rows, pubs, sample)
        total_t += dt
        total_e += e
    value = total_e / total_t
    desc = (f"one instance of each log size {logs[sample[0]]}..{logs[sample[-1]]} of the workload (its size mix; sum 2^logN = "
            f"{total_e // args.steps}), FFT + prove with the C++ oracle on {threads} threads per step")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * total_t / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32/u64",
        "data": "synthetic (seeded SplitMix64)", "config": config_block(args, logs),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": desc, "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "The reference (Swift + Metal) cannot run on Linux/B200; this arm times the repository's C++ restatement of its CPU oracles.",
    }
    print(json.dumps(line), flush=True)


def serving_mix(n_jobs, seed, lo=12, hi=22, sumcheck_every=5):
    """Job kinds and log sizes of the serving stream: commit-and-fold jobs with log
    codeword sizes in [lo, hi], P(k) proportional to 2^-(k-lo)/2, and one M31
    multilinear sum-check over 2^20 evaluations after every four of them."""
    ks = np.arange(lo, hi + 1)
    w = 2.0 ** (-(ks - lo) / 2.0)
    cdf = np.cumsum(w / w.sum())
    u = (splitmix64(seed, n_jobs) >> np.uint64(11)).astype(np.float64) / float(1 << 53)
    jobs = []
    for i in range(n_jobs):
        if i % sumcheck_every == sumcheck_every - 1:
            jobs.append(("sc", 20))
        else:
            jobs.append(("pcs", int(ks[min(len(ks) - 1, int(np.searchsorted(cdf, u[i], side="right")))])))
    return jobs


def run_serving(azk, ctx, args, batched_jobs_per_s, batched_elems_per_s=None):
    """Continuous-batching server on the serving mix.  A backlog and an overloaded
    Poisson run give the server's throughput on this mix; Poisson arrivals at
    `--serve-load` x the batched superstep's jobs/s (the 512-instance leg) give
    p50/p99 latency (completion - arrival).  Every job's bytes are those of the same
    job alone (tests/test_gpu_server.py)."""
    final_log, queries, blowup = args.final_log, 64, 2
    rng_rows = {k: None for k in range(12, 23)}
    for k in rng_rows:
        r = np.zeros(((1 << k) >> 2, 4), np.uint32)
        r[:, 0] = uniform_m31(SEED ^ (0x5E7 + k), len(r))
        rng_rows[k] = r
    sc_tables = [uniform_m31(SEED ^ (0x5C0 + i), 1 << 20) for i in range(2)]
    pubs = public_digests(4096, SEED ^ 0x5E)
    server = azk.ProofServer(ctx, hbm_budget_bytes=int(args.serve_budget_gb * (1 << 30)), slots=args.serve_slots,
                             schedule=dict(treelet_log=args.treelet_log, group_log=args.group_log, threads=args.threads, use_graph=1))

    # the job inputs are arrays that nothing changes while the server runs: they are
    # handed over without a copy (the workers read them into page-locked staging)
    def submit(job, i):
        kind, k = job
        if kind == "sc":
            return server.submit_sumcheck(sc_tables[i % 2], copy=False)
        return server.submit_pcs(k, blowup, queries, k - final_log, rng_rows[k], pubs[32 * (i % 4096):32 * (i % 4096) + 32], copy=False)

    def collect(ids):
        server.wait_all()
        return [server.poll(j) for j in ids]

    # every worker builds its device memory and pinned staging for every shape of
    # the mix before the timed runs, then a short stretch of the mix itself
    t0 = time.perf_counter()
    server.warm(pcs_shapes=[(k, k - final_log) for k in range(12, 23)], log_blowup=blowup, queries=queries, sumcheck_logs=[20])
    collect([submit(j, i) for i, j in enumerate(serving_mix(4 * args.serve_slots, SEED ^ 0x3B))])
    t_warm = time.perf_counter() - t0

    # saturated backlog: the server's throughput on this mix, the median of three
    # backlogs (each submitted at once and waited for) after one untimed backlog: a
    # fresh process's first thousands of proofs land in host memory the allocator
    # has not handed out before (page faults on every new page), which a serving
    # process does once
    mix = serving_mix(args.serve_backlog, SEED ^ 0xB1)
    collect([submit(j, i) for i, j in enumerate(mix)])
    sat_runs = []
    for _ in range(3):
        s0 = server.stats()
        t0 = time.perf_counter()
        ids = [submit(j, i) for i, j in enumerate(mix)]
        collect(ids)
        t = time.perf_counter() - t0
        sat_runs.append((t, server.stats()["pcs_elements"] - s0["pcs_elements"]))
    t_sat, sat_elems = sorted(sat_runs)[1]
    sat_jobs_s = len(mix) / t_sat
    sat_elems_s = sat_elems / t_sat
    sat_runs_jobs_s = [len(mix) / t for t, _ in sat_runs]

    def poisson(lam, seconds, seed, steady_after=0.0):
        """Submit Poisson arrivals at `lam` jobs/s for `seconds`; returns the job ids,
        submission lags and the completion rate counted from `steady_after` seconds
        into the run to its end."""
        n = max(50, int(lam * seconds))
        jobs = serving_mix(n, seed)
        gaps = -np.log1p(-((splitmix64(seed ^ 0x9A, n) >> np.uint64(11)).astype(np.float64) / float(1 << 53))) / lam
        arrivals = np.cumsum(gaps)
        ids, lags = [], []
        mark = None
        c0 = server.stats()["completed"]
        t0 = time.perf_counter()
        for i, (job, at) in enumerate(zip(jobs, arrivals)):
            while True:
                now = time.perf_counter() - t0
                if now >= at:
                    break
                if at - now > 2e-3:
                    time.sleep(at - now - 1e-3)
            if mark is None and now >= steady_after:
                mark = (server.stats()["completed"], time.perf_counter())
            ids.append(submit(job, i))
            lags.append(time.perf_counter() - t0 - at)
        c1, t1 = server.stats()["completed"], time.perf_counter()
        if mark is None:
            mark = (c0, t0)
        return jobs, ids, lags, (c1 - mark[0]) / (t1 - mark[1]), t0

    # sustained rate: arrivals above what the backlog suggests, completions counted
    # once the queue has been full for a second (a backlog of simultaneous jobs
    # reads higher than what the mix sustains under continuous arrivals)
    _, over_ids, _, sustained, _ = poisson(1.5 * sat_jobs_s, 3.0, SEED ^ 0x0F, steady_after=1.0)
    collect(over_ids)

    # Poisson arrivals at `serve_load` x the batched superstep's jobs/s (the mix's
    # sustained rate is reported beside it, so the load it puts on the server shows)
    lam = args.serve_rate if args.serve_rate > 0 else args.serve_load * batched_jobs_per_s
    s0 = server.stats()
    mix, ids, lags, _, t0 = poisson(lam, args.serve_seconds, SEED ^ 0xA7)
    res = collect(ids)
    t_run = time.perf_counter() - t0
    s1 = server.stats()
    lat = np.array([r[1] + lag for r, lag in zip(res, lags)])
    kinds = np.array([j[0] for j in mix])
    groups = server.group_stats()
    server.close()

    def pct(v):
        return {"p50_ms": float(np.percentile(v, 50) * 1e3), "p99_ms": float(np.percentile(v, 99) * 1e3), "jobs": int(len(v))} if len(v) else None

    return {
        "mix": "commit-and-fold jobs log U*[12,22] with P(k) ~ 2^-(k-12)/2 (blowup 4, fold to log 6, 64 queries) : "
               "M31 multilinear sum-check over 2^20 evaluations = 4:1",
        "slots": args.serve_slots, "hbm_budget_gb": args.serve_budget_gb, "submission": "no-copy (azk_server_submit_*_nocopy)",
        "saturated": {"jobs_per_s": sat_jobs_s, "elems_per_s": sat_elems_s, "jobs": args.serve_backlog, "seconds": t_sat,
                      "runs_jobs_per_s": sat_runs_jobs_s, "rule": "median of three backlogs after one untimed backlog"},
        "arrival_rate_jobs_per_s": lam,
        "sustained_jobs_per_s": sustained,
        "arrival_rule": f"{args.serve_load} x the batched superstep's jobs/s" if args.serve_rate <= 0 else "fixed",
        "sustained_rule": "completions in seconds 1-3 of arrivals at 1.5 x the backlog rate",
        "load_vs_sustained": lam / sustained if sustained > 0 else None,
        "batched_superstep_jobs_per_s": batched_jobs_per_s,
        "throughput_elems_per_s": (s1["pcs_elements"] - s0["pcs_elements"]) / t_run, "jobs_per_s": len(mix) / t_run,
        "latency_all": pct(lat), "latency_pcs": pct(lat[kinds == "pcs"]), "latency_sumcheck": pct(lat[kinds == "sc"]),
        "submit_lag_p99_ms": float(np.percentile(lags, 99) * 1e3), "warmup_s": t_warm,
        "held_gb": s1["held_bytes"] / 2**30,
        "pcs_groups": groups,
        "saturated_vs_batched_superstep": sat_elems_s / batched_elems_per_s if batched_elems_per_s else None,
    }


def _hashlib_merkle_check(leaf, index, siblings, root) -> bool:
    """A Merkle opening checked with Python's hashlib (independent of this library):
    SHA3-256 of the leaf, then of (left || right) up the path."""
    import hashlib

    cur = hashlib.sha3_256(leaf).digest()
    for level, sib in enumerate(siblings):
        cur = hashlib.sha3_256(cur + sib if ((index >> level) & 1) == 0 else sib + cur).digest()
    return cur == root


def run_primitives(azk, ctx, device, reps=5, seed=0xA11CE002):
    """The survey's C2/C3 primitives at full size with inputs resident in HBM
    (seeded random bytes and M31 values drawn on the device): Keccak-f[1600] over
    2^24 states, SHA3-256 over 2^24 messages of 32/64/128/136 bytes, the SHA3
    Merkle commitment of 2^24 64-byte leaves with 1024 openings, one log-22 Circle
    PCS proof (16 rounds, 64 queries), the QM31 and Circle folds of 2^24 values and
    the 2^20 multilinear sum-check.  Device time (CUDA events) is the median of
    `reps` launches after warm-up.  SHA3 digests and Merkle openings are checked
    here with hashlib on 1024 sampled items; the other rows keep samples for the
    CPU oracle, which checks them in the CPU leg."""
    import torch

    dev = torch.device("cuda", device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    n = 1 << 24
    rng = np.random.default_rng(seed)
    peak = azk.probe_int_issue(ctx) / 4320.0
    hbm, _ = measured_peaks()
    rows, samples = {}, {}

    def med(f):
        f()
        f()
        return statistics.median(f() for _ in range(reps))

    def rand_u8(count):
        return torch.randint(0, 256, (count,), dtype=torch.uint8, device=dev, generator=gen)

    # Keccak-f[1600]: 2^24 states of 200 bytes in, 200 out
    st, out = rand_u8(200 * n), torch.empty(200 * n, dtype=torch.uint8, device=dev)
    plan = azk.KeccakF1600PermutationPlan(ctx, n)
    t = med(lambda: plan.permute_resident(st.data_ptr(), out.data_ptr()).gpu_s)
    idx = np.sort(rng.choice(n, 1024, replace=False))
    ti = torch.as_tensor(idx, device=dev)
    samples["keccak"] = (st.view(n, 200)[ti].cpu().numpy(), out.view(n, 200)[ti].cpu().numpy())
    rows["keccak_f1600_2e24"] = {"seconds": t, "perms_per_s": n / t, "frac_int_roofline": n / t / peak, "hbm_gbs": 400 * n / t / 1e9}
    del st, out, plan
    # SHA3-256 of 2^24 messages per length (136 bytes take two permutations)
    import hashlib

    sha_ok = True
    for length in (32, 64, 128, 136):
        msgs, dig = rand_u8(length * n), torch.empty(32 * n, dtype=torch.uint8, device=dev)
        plan = azk.SHA3FixedOneBlockHashPlan(ctx, n, length, length)
        t = med(lambda: plan.hash_resident(msgs.data_ptr(), dig.data_ptr()).gpu_s)
        m_s, d_s = msgs.view(n, length)[ti].cpu().numpy(), dig.view(n, 32)[ti].cpu().numpy()
        ok = all(hashlib.sha3_256(m_s[k].tobytes()).digest() == d_s[k].tobytes() for k in range(len(idx)))
        sha_ok &= ok
        perms = n * (2 if length == 136 else 1)
        rows[f"sha3_256_2e24_{length}B"] = {"seconds": t, "hashes_per_s": n / t, "frac_int_roofline": perms / t / peak, "sample_equal_hashlib": ok}
        del msgs, dig, plan
    # Merkle over 2^24 x 64-byte leaves with 1024 openings
    leaves = rand_u8(64 * n)
    plan = azk.SHA3RawLeavesMerkleCommitPlan(ctx, n, 64, 64)
    root = None

    def commit():
        nonlocal root
        root = plan.commit_resident(leaves.data_ptr())
        return plan.last_stats.gpu_s

    t = med(commit)
    oidx = rng.integers(0, n, size=1024)
    paths = plan.open_resident(oidx)
    t_open = plan.last_stats.gpu_s or plan.last_stats.cpu_wall_s
    lv = leaves.view(n, 64)[torch.as_tensor(oidx, device=dev)].cpu().numpy()
    open_ok = all(_hashlib_merkle_check(lv[k].tobytes(), int(oidx[k]), paths[k], root) for k in range(len(oidx)))
    rows["merkle_2e24_64B"] = {"seconds": t, "perms_per_s": (2 * n - 1) / t, "frac_int_roofline": (2 * n - 1) / t / peak,
                               "openings": 1024, "openings_s": t_open, "openings_verify_hashlib": open_ok}
    del leaves, plan
    # one log-22 PCS proof from coefficients (blowup 4, 16 rounds, 64 queries)
    lg = 22
    coeffs = np.zeros(((1 << lg) >> 2, 4), np.uint32)
    coeffs[:, 0] = uniform_m31(seed ^ 0xC3, len(coeffs))
    pub = public_digests(1, seed ^ 0xC3)
    prover = azk.CirclePCSFRIProver(ctx, lg, 2, 64, 16)
    proof = None

    def prove():
        nonlocal proof
        proof = prover.prove_coefficients(coeffs, pub)
        return prover.last_stats.gpu_s

    t = med(prove)
    perms = sum(2 * ((1 << lg) >> k) - 1 + 3 for k in range(16))
    samples["c3"] = (coeffs, pub, proof)
    rows["pcs_prove_log22"] = {"seconds": t, "elems_per_s": (1 << lg) / t, "frac_int_roofline": perms / t / peak, "proof_bytes": len(proof),
                               "wall_s": prover.last_stats.cpu_wall_s}
    del prover
    # QM31 fold of 2^24 values with QM31 inverse points (16n + 8n read, 8n write)
    ev = torch.randint(0, 2**31 - 1, (n * 4,), dtype=torch.int32, device=dev, generator=gen)
    inv = torch.randint(1, 2**31 - 1, (n * 2,), dtype=torch.int32, device=dev, generator=gen)
    fo = torch.empty(n * 2, dtype=torch.int32, device=dev)
    ch = np.array([[11, 13, 17, 19]], np.uint32)
    fplan = azk.QM31FRIFoldPlan(ctx, n)
    t = med(lambda: fplan.execute_resident(ev.data_ptr(), inv.data_ptr(), fo.data_ptr(), ch).gpu_s)
    fidx = torch.as_tensor(idx[:256] // 2, device=dev)
    samples["fold"] = (ev.view(n // 2, 8)[fidx].cpu().numpy().view(np.uint32), inv.view(n // 2, 4)[fidx].cpu().numpy().view(np.uint32),
                       fo.view(n // 2, 4)[fidx].cpu().numpy().view(np.uint32), ch)
    rows["qm31_fold_2e24"] = {"seconds": t, "hbm_gbs": 32 * n / t / 1e9, "frac_hbm": 32 * n / t / 1e9 / hbm,
                              "algorithmic": "16n + 8n read + 8n write bytes (n inputs)"}
    del ev, inv, fo, fplan
    # Circle FFT stage of 16 log-22 instances (blowup 4) inside the batched superstep:
    # lifted M31 coefficients (one-limb tiles) and full QM31 coefficients (QM31
    # tiles); bytes: 16 per nonzero coefficient read, 16N written, 4(N-1) twiddles
    lg, cnt = 22, 16
    rows_n = (1 << lg) >> 2
    for label, limbs in (("m31", 1), ("qm31", 4)):
        flat = np.zeros((rows_n * cnt, 4), np.uint32)
        flat[:, :limbs] = uniform_m31(seed ^ (0xF0 + limbs), rows_n * cnt * limbs).reshape(rows_n * cnt, limbs)
        pubs = public_digests(cnt, seed ^ (0xF0 + limbs))
        b = azk.BatchProver(ctx, [lg] * cnt, [lg - 6] * cnt, 2, 64)
        b.upload(flat, [rows_n * i for i in range(cnt)], [rows_n] * cnt)
        b.prove(pubs)
        b.set_profiling(True)
        fs = []
        for _ in range(reps):
            b.prove(pubs)
            fs.append(b.profile()["fft_s"])
        t = statistics.median(fs)
        N = 1 << lg
        alg = cnt * (16 * rows_n + 16 * N + 4 * (N - 1))
        rows[f"circle_fft_16x_log22_{label}"] = {"seconds": t, "elems_per_s": cnt * N / t, "hbm_gbs": alg / t / 1e9, "frac_hbm": alg / t / 1e9 / hbm,
                                                 "algorithmic": "16 B per nonzero coefficient + 16N written + 4(N-1) twiddle bytes per codeword"}
        if limbs == 4:
            samples["fft_qm31"] = (flat[:rows_n].copy(), pubs[:32], b.proofs()[0])
        del b, flat
    # M31 multilinear sum-check of 2^20 evaluations (sequential digest + 20 rounds)
    sc = uniform_m31(seed ^ 0x5C, 1 << 20)
    res = None

    def sumcheck():
        nonlocal res
        t0 = time.perf_counter()
        res = azk.sumcheck_prove(ctx, sc)
        return time.perf_counter() - t0

    t = med(sumcheck)
    samples["sumcheck"] = (sc, res)
    perms = (50 + 4 * len(sc)) // 136 + 1
    rows["sumcheck_2e20"] = {"wall_s": t, "seconds": res["gpu_s"], "digest_permutations": perms, "us_per_permutation": res["gpu_s"] / perms * 1e6}
    torch.cuda.empty_cache()  # give the device memory of the inputs back before serving
    return {"rows": rows, "int_peak_perms_per_s": peak, "hbm_peak_gbs": hbm,
            "checks_here": {"sha3_sample_equal_hashlib": sha_ok, "merkle_openings_verify_hashlib": open_ok}}, samples


def check_primitive_samples(samples) -> dict:
    """The CPU oracle on the primitives' samples (runs in the CPU leg)."""
    from oracle import pyoracle as O

    out = {}
    if "keccak" in samples:
        s_in, s_out = samples["keccak"]
        out["keccak_sample_equal"] = bool(np.array_equal(O.keccak_f1600(s_in.reshape(-1)).reshape(s_out.shape), s_out))
    if "fold" in samples:
        ev, inv, got, ch = samples["fold"]
        want = np.stack([O.fold(ev[k].reshape(2, 4), inv[k:k + 1], ch[0])[0] for k in range(len(ev))])
        out["qm31_fold_sample_equal"] = bool(np.array_equal(want, got))
    if "c3" in samples:
        coeffs, pub, proof = samples["c3"]
        full = np.zeros((1 << 22, 4), np.uint32)
        full[: len(coeffs)] = coeffs
        r = O.prove(22, O.fft_evaluate(22, full), 2, 64, pub, 16)
        out["pcs_log22_proof_equal"] = r.proof == proof
        out["pcs_log22_verified"] = O.verify(proof, pub)
    if "fft_qm31" in samples:
        coeffs, pub, proof = samples["fft_qm31"]
        full = np.zeros((1 << 22, 4), np.uint32)
        full[: len(coeffs)] = coeffs
        out["fft_qm31_proof_equal"] = O.prove(22, O.fft_evaluate(22, full), 2, 64, pub, 16).proof == proof
    if "sumcheck" in samples:
        ev, res = samples["sumcheck"]
        want = O.sumcheck_multilinear(ev)
        out["sumcheck_equal"] = (res["claimed_sum"] == want["claimed_sum"] and res["final"] == want["final"]
                                 and res["initial_digest"] == want["initial_digest"] and np.array_equal(res["challenges"], want["challenges"]))
    return out


def plain_values_ok(v):
    return v is not None and v > 0


METRIC = "commit+FRI-fold M31 elems/s batched vs plain on 1 B200, bit-exact; p50/p99"
UNIT = "elems/s"


def config_block(args, logs):
    return {
        "workload": f"{len(logs)} Circle PCS/FRI commit-and-fold instances, log sizes U[{args.lo},{args.hi}] (seed 0xA11CE004), blowup 4, "
                    f"16-B QM31 leaves, fold to log {args.final_log}, 64 queries, proof bytes on device",
        "instances": len(logs),
        "total_codeword_elems": int(sum(1 << lg for lg in logs)),
        "schedule": ({"treelet_log": args.treelet_log, "group_log": args.group_log, "threads": args.threads or 256, "graph": True} if args.treelet_log else
                     {"treelet": "tuned per-layer table (cost model over measured timings, csrc/azk_tuned.h pcs_batch)", "group_log": args.group_log,
                      "threads": args.threads or "tuned per-layer table (pcs_batch: 256)", "graph": True}),
        "l2": "inputs larger than L2 (codewords and trees of one superstep are several GB)",
        "parallelism": f"replicas x{int(os.environ.get('WORLD_SIZE', '1'))} (no data-path collective)",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--lo", type=int, default=10)
    ap.add_argument("--hi", type=int, default=22)
    ap.add_argument("--final-log", type=int, default=6)
    ap.add_argument("--treelet-log", type=int, default=0, help="fixed treelet depth (0: the library's tuned per-layer table)")
    ap.add_argument("--compare-schedules", type=int, default=1)
    ap.add_argument("--leaf64", type=int, default=1)
    ap.add_argument("--group-log", type=int, default=12)
    ap.add_argument("--threads", type=int, default=0, help="threads per CTA of the commit kernel (0: the tuned per-layer tables)")
    ap.add_argument("--plain-steps", type=int, default=5)
    ap.add_argument("--plain-warmup", type=int, default=1)
    ap.add_argument("--cpu-max-log", type=int, default=64, help="largest log size in the CPU oracle's sample")
    ap.add_argument("--tuner-ab", type=int, default=1, help="time the plain form and single trees at a fixed depth beside the tuned tables")
    ap.add_argument("--primitives", type=int, default=1, help="measure the C2/C3 primitives at full size (outputs sample-checked)")
    ap.add_argument("--literal-max-log", type=int, default=14, help="largest log size the literal single-thread CPU form proves")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--e2e-pipeline", type=int, default=1)
    ap.add_argument("--serve-slots", type=int, default=32)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--serve-backlog", type=int, default=1000)
    ap.add_argument("--serve-load", type=float, default=0.8)
    ap.add_argument("--serve-seconds", type=float, default=5.0)
    ap.add_argument("--serve-rate", type=float, default=0.0, help="fixed arrival rate (jobs/s) instead of the load rule")
    args = ap.parse_args()

    world, rank, local, dist = dist_setup(args)
    logs, rounds, counts, offsets = workload(args.instances, args.lo, args.hi, args.final_log)
    rows = coefficient_rows(counts)
    pubs = public_digests(len(logs))
    if args.impl == "reference":
        run_reference(args, logs, rounds, counts, offsets, rows, pubs, world, rank, dist)
        if dist is not None:
            dist.destroy_process_group()
        return

    import apple_b200 as azk

    ctx = azk.Context(local)
    # schedule: the library's tuned per-layer table for batched supersteps unless a
    # fixed treelet depth is asked for
    if args.treelet_log:
        sched = dict(treelet_log=args.treelet_log, group_log=args.group_log, threads=args.threads or 256, use_graph=1)
    else:
        sched = dict(group_log=args.group_log, threads=args.threads, use_graph=1)
    batch = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=sched)
    work = batch.work()
    elems = int(sum(1 << lg for lg in logs))

    # pinned host staging for the end-to-end path
    import torch

    pinned = torch.empty((rows.shape[0], 4), dtype=torch.int32, pin_memory=True)
    pinned.numpy().view(np.uint32)[:] = rows
    host_rows = pinned.numpy().view(np.uint32)
    proof_host = torch.empty(max(1, batch.proof_total), dtype=torch.uint8, pin_memory=True)

    batch.upload(host_rows, offsets, counts)
    for _ in range(args.warmup):
        batch.prove(pubs)

    # ---- device-timed batched superstep ----
    clocks = ClockSampler(local)
    clocks.start()
    barrier(dist)
    gpu_times = []
    for _ in range(args.steps):
        st = batch.prove(pubs)
        gpu_times.append(st.gpu_s)
    barrier(dist)
    clk = clocks.stop()
    t_dev = max_over_ranks(dist, sum(gpu_times), local)
    value = world * elems * args.steps / t_dev
    print(f"[bench] batched steps: {[round(1000 * g, 2) for g in gpu_times]} ms", file=sys.stderr, flush=True)
    # the proofs of the last timed superstep, checked against the oracle below
    gpu_proofs = batch.proofs() if rank == 0 and not args.no_cpu else None

    # ---- per-stage profile (events inside the captured graph) ----
    batch.set_profiling(True)
    batch.prove(pubs)
    prof = batch.profile()
    batch.set_profiling(False)

    # ---- end to end through the C ABI from pinned host memory ----
    h2d = int(sum(counts)) * 16
    d2h = batch.proof_total
    e2e_times = []
    import ctypes

    for _ in range(max(1, args.steps // 2)):
        t0 = time.perf_counter()
        batch.upload(host_rows, offsets, counts)
        batch.prove(pubs)
        azk._capi.check(azk.lib().azk_batch_download_proofs(batch._h, ctypes.c_void_p(proof_host.data_ptr()), batch.proof_total), ctx.handle)
        e2e_times.append(time.perf_counter() - t0)
    t_e2e = max_over_ranks(dist, statistics.median(e2e_times), local)
    e2e_serial = world * elems / t_e2e

    # ---- pipelined end to end: two provers alternate, so one step's copies
    # overlap the other's kernels (every step still uploads its inputs from
    # pinned host memory and reads its proofs back) ----
    e2e_pipe = None
    if args.e2e_pipeline:
        batch2 = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=sched)
        batch2.upload(host_rows, offsets, counts)
        batch2.prove(pubs)
        proof_host2 = torch.empty(max(1, batch.proof_total), dtype=torch.uint8, pin_memory=True)
        per_lane = max(2, (args.steps + 1) // 2)
        errors = []
        # Two-stage pipeline: the supersteps take turns on the GPU (one prover
        # proves while the other downloads its proofs and uploads its next inputs).
        # Run side by side instead, two supersteps share the GPU, finish together
        # and then both copy while the GPU idles.
        gpu_turn = threading.Lock()
        lanes = [(batch, proof_host), (batch2, proof_host2)]

        def lane(b, ph):
            try:
                for _ in range(per_lane):
                    b.upload(host_rows, offsets, counts)
                    with gpu_turn:
                        b.prove(pubs)
                    azk._capi.check(azk.lib().azk_batch_download_proofs(b._h, ctypes.c_void_p(ph.data_ptr()), b.proof_total), ctx.handle)
            except Exception as exc:  # surfaced below
                errors.append(exc)

        barrier(dist)
        t0 = time.perf_counter()
        threads = [threading.Thread(target=lane, args=ln) for ln in lanes]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        t_pipe = time.perf_counter() - t0
        if errors:
            raise errors[0]
        t_pipe = max_over_ranks(dist, t_pipe / (2 * per_lane), local)
        e2e_pipe = world * elems / t_pipe
        del batch2, lanes, threads
    e2e_value = e2e_pipe if e2e_pipe else e2e_serial
    t_e2e_report = world * elems / e2e_value

    proof_total = batch.proof_total

    # ---- the commit launches as persistent work-queue grids instead of one CTA per
    # treelet (same schedule otherwise) ----
    persistent = None
    if args.compare_schedules:
        bqp = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=dict(sched, persistent_trees=1))
        bqp.upload(host_rows, offsets, counts)
        bqp.prove(pubs)
        ptq = [bqp.prove(pubs).gpu_s for _ in range(3)]
        del bqp
        t_pq = max_over_ranks(dist, statistics.median(ptq), local)
        persistent = {"value": world * elems / t_pq, "unit": UNIT, "ms_per_step": 1000 * t_pq,
                      "over_static_grid": (world * elems / t_pq) / value,
                      "schedule": "each round's commit launch a grid of the resident CTAs pulling treelets from a device counter"}

    # ---- the same superstep with one fixed treelet depth everywhere (the schedule
    # without the tuner), and the plain per-instance form on its own best schedule
    # (the single-instance tuned table) ----
    untuned_value = None
    if args.compare_schedules and not args.treelet_log:
        del batch
        batch = None
        bu = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=dict(treelet_log=12, group_log=12, threads=256, use_graph=1))
        bu.upload(host_rows, offsets, counts)
        bu.prove(pubs)
        ut = [bu.prove(pubs).gpu_s for _ in range(2)]
        untuned_value = world * elems / max_over_ranks(dist, statistics.median(ut), local)
        del bu
    plain_times = []
    plain_mismatch = False
    if args.plain_steps:
        tables = tuned_tables()
        thr = tuned_thread_tables() or {}
        psched = dict(layer_treelet=tables["pcs_single"], group_log=args.group_log, threads=args.threads, use_graph=0) if tables and not args.treelet_log \
            else sched
        if psched is not sched and not args.threads and "pcs_single" in thr:
            psched["layer_threads"] = thr["pcs_single"]
        if batch is not None:
            del batch
            batch = None
        bp = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=psched)
        bp.upload(host_rows, offsets, counts)
        for _ in range(args.plain_warmup):
            bp.prove(pubs, plain=True)
        for _ in range(args.plain_steps):
            st = bp.prove(pubs, plain=True)
            plain_times.append(st.gpu_s)
        if gpu_proofs is not None and bp.proofs() != gpu_proofs:
            plain_mismatch = True
        del bp
    t_plain = max_over_ranks(dist, statistics.median(plain_times), local) if plain_times else float("nan")

    # ---- where the tuned tables matter: the plain form at one fixed depth, and
    # single fold-and-commit trees of 2^12 ... 2^16 leaves (the server's typical
    # layers), tuned depth and threads against depth 12 at 256 threads ----
    tuner_ab = None
    if args.tuner_ab and not args.treelet_log:
        from apple_b200 import autotune as T

        tables = tuned_tables() or {}
        bq = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=dict(treelet_log=12, group_log=args.group_log, threads=256, use_graph=0))
        bq.upload(host_rows, offsets, counts)
        bq.prove(pubs, plain=True)
        pt = [bq.prove(pubs, plain=True).gpu_s for _ in range(3)]
        del bq
        t_plain12 = max_over_ranks(dist, statistics.median(pt), local)
        trees = {}
        single = tables.get("pcs_single", {})
        single_threads = (tuned_thread_tables() or {}).get("pcs_single", {})
        for lg in range(12, 17):
            tl, th = int(single.get(lg, 12)), int(single_threads.get(lg, 0) or 256)
            t_tuned = T.time_tree(ctx, lg, 16, 1, 1, tl, th, reps=7)
            t_fixed = T.time_tree(ctx, lg, 16, 1, 1, min(12, lg), 256, reps=7)
            trees[lg] = {"tuned": [tl, th], "tuned_us": 1e6 * t_tuned, "depth12_us": 1e6 * t_fixed, "tuned_over_depth12": t_fixed / t_tuned}
        tuner_ab = {"plain_depth12_ms": 1000 * t_plain12, "plain_tuned_over_depth12": t_plain12 / t_plain if plain_times else None,
                    "single_trees": trees,
                    "note": "device time of one fold-and-commit tree of 2^k 16-byte leaves (median of 7); plain form: whole superstep, median of 3"}

    # ---- the same superstep with 64-byte Merkle leaves (4 QM31 per leaf): the
    # survey's second C4 row; bit-exact against the oracle's 64-byte-leaf chain, no
    # verifier proof format ----
    leaf64 = None
    if args.leaf64:
        b64 = azk.BatchProver(ctx, logs, rounds, 2, 64, schedule=sched, leaf_bytes=64)
        b64.upload(host_rows, offsets, counts)
        for _ in range(args.warmup):
            b64.prove(pubs)
        lt = [b64.prove(pubs).gpu_s for _ in range(max(2, args.steps // 2))]
        t64 = max_over_ranks(dist, statistics.median(lt), local)
        w64 = b64.work()
        leaf64 = {"value": world * elems / t64, "unit": UNIT, "ms_per_step": 1000 * t64, "tree_permutations": w64["tree_permutations"],
                  "output": "commitments, challenges, final layers (no proof encoding: the reference's verifier opens 16-byte leaves)"}
        del b64
    print(f"[bench] plain: {[round(1000 * g, 2) for g in plain_times]} ms, e2e {[round(1000 * g, 2) for g in e2e_times]} ms, profile {prof}",
          file=sys.stderr, flush=True)
    plain_value = world * elems / t_plain if plain_times else None

    # ---- rooflines ----
    int_ops = azk.probe_int_issue(ctx)
    perm_peak = int_ops / 4320.0
    tree_rate = work["tree_permutations"] / prof["tree_s"] if prof["tree_s"] > 0 else 0.0
    tree_launches = max(1, max(rounds))
    hbm_gbs, hbm_kind = measured_peaks()
    # FFT bytes: the input's nonzero prefix (16 B per coefficient read; the zero tail
    # is known from the upload and never read) + the 16 B per element codeword
    # written + 4 B per stage twiddle; the dense figure charges all 16N input bytes
    fft_bytes_prefix = int(sum(16 * c + 16 * (1 << lg) + 4 * ((1 << lg) - 1) for c, lg in zip(counts, logs)))
    fft_gbs = fft_bytes_prefix / prof["fft_s"] / 1e9 if prof["fft_s"] > 0 else 0.0
    fft_gbs_dense = work["fft_bytes"] / prof["fft_s"] / 1e9 if prof["fft_s"] > 0 else 0.0
    traffic = profile_traffic()

    primitives, prim_samples = None, {}
    if args.primitives and world == 1:
        primitives, prim_samples = run_primitives(azk, ctx, local)
        print(f"[bench] primitives {primitives}", file=sys.stderr, flush=True)

    serving = None
    if not args.no_serve and world == 1:
        serving = run_serving(azk, ctx, args, len(logs) * args.steps / t_dev, value / world)
        print(f"[bench] serving {serving}", file=sys.stderr, flush=True)

    line = None
    parity_ok = True
    if rank == 0:
        cpu = None
        parity = None
        if not args.no_cpu and world == 1:
            from oracle import pyoracle as O

            sample = stratified_sample(logs, args.cpu_max_log)
            e, dt, want = cpu_sample(logs, rounds, counts, offsets, rows, pubs, sample)
            equal = [i for i in sample if gpu_proofs[i] == want[i]]
            t0 = time.perf_counter()
            accepted = verify_all(gpu_proofs, pubs)
            t_verify = time.perf_counter() - t0
            parity = {"instances_checked": len(sample), "equal": len(equal) == len(sample), "log_sizes": [logs[i] for i in sample],
                      "verified": int(sum(accepted)), "verified_of": len(gpu_proofs), "verified_all": all(accepted),
                      "plain_equal": not plain_mismatch, "verify_s": t_verify,
                      "check": "proof bytes of the stratified sample equal the oracle's; every proof of the superstep is accepted by "
                               "the oracle's verifier; the plain form's proofs equal the batched form's"}
            parity_ok = parity["equal"] and parity["verified_all"] and not plain_mismatch
            if primitives is not None:
                primitives["checks_oracle"] = check_primitive_samples(prim_samples)
                prim_ok = all(primitives["checks_oracle"].values()) and all(primitives["checks_here"].values())
                parity["primitives_equal"] = prim_ok
                parity_ok = parity_ok and prim_ok
            cpu = {"value": e / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port", "cpu_model": cpu_model(),
                   "sample": f"one instance of each log size {logs[sample[0]]}..{logs[sample[-1]]} of the workload (its size mix; "
                             f"sum 2^logN = {e}), FFT + prove with the C++ oracle on {O.num_threads()} threads ({dt:.1f} s)"}
            if args.literal_max_log:
                le, ldt, lproofs = cpu_literal_sample(logs, rounds, counts, offsets, rows, pubs, args.literal_max_log)
                if lproofs:
                    cpu["literal_single_thread"] = {
                        "value": le / ldt, "unit": UNIT, "cores": 1, "seconds": ldt, "log_sizes": [logs[i] for i in lproofs],
                        "equal": all(lproofs[i] == gpu_proofs[i] for i in lproofs),
                        "form": "the reference's literal builder: one thread, radix-2 FFT stage by stage, a full layer re-hash "
                                "for every opening, the transcript replayed from the start for every challenge; sizes above "
                                f"log {args.literal_max_log} are not run (the per-opening rebuild grows as queries x rounds x N)"}
                    parity["equal"] = parity["equal"] and cpu["literal_single_thread"]["equal"]
                    parity_ok = parity_ok and cpu["literal_single_thread"]["equal"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000 * t_dev / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u32/u64 (M31/QM31 field, Keccak lanes)", "data": "synthetic (seeded SplitMix64)", "config": config_block(args, logs),
            "parity": parity,
            "plain": {"value": plain_value, "unit": UNIT, "ms_per_step": 1000 * t_plain if plain_values_ok(plain_value) else None,
                      "samples_ms": [1000 * t for t in plain_times], "warmup": args.plain_warmup,
                      "spread_ms": [1000 * min(plain_times), 1000 * max(plain_times)] if plain_times else None,
                      "batched_over_plain": value / plain_value if plain_values_ok(plain_value) else None,
                      "schedule": "tuned single-instance per-layer table" if (tuned_tables() and not args.treelet_log) else "same as batched"},
            "leaf64": leaf64,
            "untuned": {"value": untuned_value, "unit": UNIT, "schedule": "treelet depth 12 on every layer",
                        "tuned_over_untuned": value / untuned_value if untuned_value else None},
            "tuner_ab": tuner_ab,
            "persistent_trees": persistent,
            "primitives": primitives,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": 1000 * t_e2e_report,
                    "mode": "two provers taking turns on the GPU (one prover's copies overlap the other's superstep; the first upload and the last download are inside the timed region)" if e2e_pipe else "serial",
                    "serial_value": e2e_serial, "serial_ms_per_step": 1000 * t_e2e},
            "roofline": {
                "bound": "int32-issue", "kernel": "tree_tiles_kernel (fold + leaf hash + treelet + upper tree + transcript)",
                "achieved": tree_rate / 1e9, "peak": perm_peak / 1e9, "unit": "Gperm/s", "frac": tree_rate / perm_peak if perm_peak else None,
                "traffic": traffic.get("tree_bytes_per_launch"),
                "peak_source": f"probe: {int_ops / 1e12:.2f} T LOP3+SHF ops/s / 4320 ops per Keccak-f",
                "algorithmic": f"{work['tree_permutations']} permutations per superstep over {tree_launches} launches",
            },
            "roofline_hbm": {
                "bound": "hbm", "kernel": "Circle FFT stage (fft_m31_tile_kernel high-stage pass + fft_m31_low_tma_kernel low-stage pass; fft_pass_m31_kernel below 2^12)", "achieved": fft_gbs, "peak": hbm_gbs,
                "unit": "GB/s",
                "frac": fft_gbs / hbm_gbs if hbm_gbs else None, "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm_kind == "measured" else "fallback 6,650 GB/s (no MEASURED_PEAKS.json)",
                "algorithmic": "16 B per nonzero input coefficient read + 16N codeword bytes written + 4(N-1) twiddle bytes per codeword",
                "algorithmic_bytes": fft_bytes_prefix,
                "dense": {"achieved": fft_gbs_dense, "frac": fft_gbs_dense / hbm_gbs if hbm_gbs else None,
                          "algorithmic": "16N read + 16N write + 4(N-1) twiddle bytes per codeword"},
                "traffic": traffic.get("fft_bytes_per_stage"),
                "traffic_scope": "DRAM bytes of the whole FFT stage of one superstep (both pass launches), like achieved",
            },
            "stage_seconds": prof,
            "gpu_launches": work["launches"] * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
            "proof_bytes_per_step": proof_total,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    if not parity_ok:
        # the reference's bench exits 2 when a GPU result differs from its CPU oracle
        print("[bench] PARITY FAILURE: GPU proofs differ from the CPU oracle", file=sys.stderr, flush=True)
        sys.exit(2)


if __name__ == "__main__":
    main()
