"""GPU: the continuous-batching server returns, for every job of a mixed stream
(Circle PCS proofs of uneven sizes and M31 multilinear sum-checks), exactly the
result the same job gives alone, admits jobs under its HBM budget and refuses a
job larger than the budget."""
import time

import numpy as np
import pytest

import apple_b200 as azk

pytestmark = pytest.mark.gpu
P = (1 << 31) - 1


def _pcs_job(rng, log_size):
    rounds = min(8, log_size)
    count = 1 << (log_size - 2)
    coeffs = rng.integers(0, P, (count, 4), dtype=np.uint32)
    pub = rng.integers(0, 256, 32, dtype=np.uint8).tobytes()
    return dict(kind="pcs", log_size=log_size, rounds=rounds, queries=32, coeffs=coeffs, pub=pub)


def _wait(server, ids, timeout=120.0):
    out, t0 = {}, time.time()
    while len(out) < len(ids):
        for j in ids:
            if j not in out:
                r = server.poll(j)
                if r is not None:
                    out[j] = r
        assert time.time() - t0 < timeout
        time.sleep(0.001)
    return out


def test_mixed_stream_matches_alone(ctx, oracle):
    rng = np.random.default_rng(0x5E4)
    jobs = []
    for k in range(20):
        if k % 5 == 4:
            jobs.append(dict(kind="sc", ev=rng.integers(0, P, 1 << int(rng.integers(10, 17)), dtype=np.uint32)))
        else:
            jobs.append(_pcs_job(rng, int(rng.integers(10, 19))))
    server = azk.ProofServer(ctx, hbm_budget_bytes=8 << 30, slots=4)
    ids = []
    for j in jobs:
        if j["kind"] == "pcs":
            ids.append(server.submit_pcs(j["log_size"], 2, j["queries"], j["rounds"], j["coeffs"], j["pub"]))
        else:
            ids.append(server.submit_sumcheck(j["ev"]))
    res = _wait(server, ids)
    server.wait_all()
    st = server.stats()
    assert st["completed"] == len(jobs)
    server.close()
    for j, i in zip(jobs, ids):
        got, lat = res[i]
        assert lat > 0
        if j["kind"] == "pcs":
            alone = azk.CirclePCSFRIProver(ctx, j["log_size"], 2, j["queries"], j["rounds"]).prove_coefficients(j["coeffs"], j["pub"])
            assert got == alone
            assert oracle.verify(got, j["pub"])
        else:
            alone = azk.sumcheck_prove(ctx, j["ev"])
            for key in ("claimed_sum", "final", "initial_digest"):
                assert got[key] == alone[key]
            for key in ("r0", "r1", "challenges"):
                assert np.array_equal(got[key], alone[key])


def test_pcs_job_matches_oracle_proof(ctx, oracle):
    rng = np.random.default_rng(7)
    j = _pcs_job(rng, 12)
    server = azk.ProofServer(ctx, hbm_budget_bytes=1 << 30, slots=2)
    jid = server.submit_pcs(12, 2, j["queries"], j["rounds"], j["coeffs"], j["pub"])
    (proof, _), = _wait(server, [jid]).values()
    server.close()
    full = np.zeros((1 << 12, 4), np.uint32)
    full[:len(j["coeffs"])] = j["coeffs"]
    ev = oracle.fft_evaluate(12, full)
    assert proof == oracle.prove(12, ev, 2, j["queries"], j["pub"], j["rounds"]).proof


def test_budget_admission_and_refusal(ctx):
    rng = np.random.default_rng(11)
    # one log-16 PCS shape is about 7.5 MiB: a 12 MiB budget runs one at a time
    server = azk.ProofServer(ctx, hbm_budget_bytes=12 << 20, slots=4)
    with pytest.raises(azk.AZKError) as e:
        server.submit_pcs(20, 2, 32, 8, rng.integers(0, P, (16, 4), dtype=np.uint32), bytes(32))
    assert e.value.name == "hbmBudget"
    jobs = [_pcs_job(rng, 16) for _ in range(6)]
    ids = [server.submit_pcs(16, 2, j["queries"], j["rounds"], j["coeffs"], j["pub"]) for j in jobs]
    res = _wait(server, ids)
    assert server.stats()["held_bytes"] <= 12 << 20
    server.close()
    for j, i in zip(jobs, ids):
        assert res[i][0] == azk.CirclePCSFRIProver(ctx, 16, 2, j["queries"], j["rounds"]).prove_coefficients(j["coeffs"], j["pub"])


def test_bad_jobs_are_refused_at_submission(ctx):
    server = azk.ProofServer(ctx, hbm_budget_bytes=1 << 30, slots=1)
    with pytest.raises(azk.AZKError):
        server.submit_sumcheck(np.zeros(3, np.uint32))
    with pytest.raises(azk.AZKError):
        server.submit_pcs(10, 2, 8, 4, np.full((4, 4), P, np.uint32), bytes(32))
    server.close()


def test_warm_then_jobs_match_alone(ctx):
    """Warm-up runs a job of zeros per shape on every worker and leaves no result
    behind; jobs of those shapes afterwards give the bytes the same job gives alone,
    and a shape over the budget is skipped rather than refused."""
    rng = np.random.default_rng(0x3A)
    server = azk.ProofServer(ctx, hbm_budget_bytes=256 << 20, slots=3)
    server.warm(pcs_shapes=[(12, 8), (14, 8), (24, 8)], log_blowup=2, queries=32, sumcheck_logs=[12])
    st = server.stats()
    assert st["completed"] == 0
    assert 0 < st["held_bytes"] <= 256 << 20
    jobs = [_pcs_job(rng, 12), _pcs_job(rng, 14), _pcs_job(rng, 12)]
    ev = rng.integers(0, P, 1 << 12, dtype=np.uint32)
    ids = [server.submit_pcs(j["log_size"], 2, j["queries"], j["rounds"], j["coeffs"], j["pub"]) for j in jobs]
    sid = server.submit_sumcheck(ev)
    res = _wait(server, ids + [sid])
    assert server.stats()["completed"] == 4
    server.close()
    for j, i in zip(jobs, ids):
        assert res[i][0] == azk.CirclePCSFRIProver(ctx, j["log_size"], 2, j["queries"], j["rounds"]).prove_coefficients(j["coeffs"], j["pub"])
    alone = azk.sumcheck_prove(ctx, ev)
    assert res[sid][0]["initial_digest"] == alone["initial_digest"]
    assert np.array_equal(res[sid][0]["challenges"], alone["challenges"])


def _shape_bytes(ctx, log_size, rounds, queries):
    """Device bytes the server holds for one PCS shape (one worker, warmed)."""
    s = azk.ProofServer(ctx, hbm_budget_bytes=1 << 34, slots=1)
    s.warm(pcs_shapes=[(log_size, rounds)], log_blowup=2, queries=queries)
    held = s.stats()["held_bytes"]
    s.close()
    return held


def test_idle_workers_give_back_memory_for_a_larger_job(ctx):
    """Shapes cached by idle workers are evicted to admit a job that does not fit
    otherwise: with a budget of one log-16 shape plus 1 MiB, workers that cached
    log-14 and log-15 shapes while those jobs ran must give all of it back for the
    log-16 job (a worker that could only drop its own cache would wait forever)."""
    rng = np.random.default_rng(0xE71C)
    a, b, c = (_shape_bytes(ctx, lg, 8, 32) for lg in (14, 15, 16))
    assert a + b < c
    server = azk.ProofServer(ctx, hbm_budget_bytes=c + (1 << 20), slots=3)
    small = [_pcs_job(rng, lg) for lg in (14, 15, 14, 15, 14, 15)]
    ids = [server.submit_pcs(j["log_size"], 2, j["queries"], j["rounds"], j["coeffs"], j["pub"]) for j in small]
    first = _wait(server, ids)
    assert server.stats()["held_bytes"] > 0
    big = _pcs_job(rng, 16)
    bid = server.submit_pcs(16, 2, big["queries"], big["rounds"], big["coeffs"], big["pub"])
    got = _wait(server, [bid], timeout=60.0)
    assert server.stats()["held_bytes"] <= c + (1 << 20)
    server.close()
    assert got[bid][0] == azk.CirclePCSFRIProver(ctx, 16, 2, big["queries"], big["rounds"]).prove_coefficients(big["coeffs"], big["pub"])
    for j, i in zip(small, ids):
        assert first[i][0] == azk.CirclePCSFRIProver(ctx, j["log_size"], 2, j["queries"], j["rounds"]).prove_coefficients(j["coeffs"], j["pub"])


def test_queued_jobs_of_one_shape_are_proved_as_one_group(ctx, oracle):
    """Same-shape PCS jobs waiting together are taken as one group and proved by one
    batched superstep; every job's proof is still the one it gives alone, and a job
    of another shape queued among them keeps its own bytes."""
    rng = np.random.default_rng(0x6A0)
    server = azk.ProofServer(ctx, hbm_budget_bytes=4 << 30, slots=1)
    jobs = [_pcs_job(rng, 12) for _ in range(12)] + [_pcs_job(rng, 14)] + [_pcs_job(rng, 12) for _ in range(5)]
    ids = [server.submit_pcs(j["log_size"], 2, j["queries"], j["rounds"], j["coeffs"], j["pub"]) for j in jobs]
    sc = rng.integers(0, P, 1 << 12, dtype=np.uint32)
    sid = server.submit_sumcheck(sc)
    res = _wait(server, ids + [sid])
    gs = server.group_stats()
    server.close()
    assert gs["grouped_jobs"] == len(jobs) and gs["groups"] < len(jobs)
    for j, i in zip(jobs, ids):
        assert res[i][0] == azk.CirclePCSFRIProver(ctx, j["log_size"], 2, j["queries"], j["rounds"]).prove_coefficients(j["coeffs"], j["pub"])
    full = np.zeros((1 << 12, 4), np.uint32)
    full[: len(jobs[0]["coeffs"])] = jobs[0]["coeffs"]
    assert res[ids[0]][0] == oracle.prove(12, oracle.fft_evaluate(12, full), 2, jobs[0]["queries"], jobs[0]["pub"], jobs[0]["rounds"]).proof
    want = oracle.sumcheck_multilinear(sc)
    assert res[sid][0]["initial_digest"] == want["initial_digest"] and np.array_equal(res[sid][0]["challenges"], want["challenges"])


def test_sumcheck_lane_batches_many_tables(ctx, oracle):
    """Many sum-check tables in flight at once (several per batched launch) each give
    the oracle's proof."""
    rng = np.random.default_rng(0x5C5)
    server = azk.ProofServer(ctx, hbm_budget_bytes=4 << 30, slots=2)
    tables = [rng.integers(0, P, 1 << int(rng.integers(8, 15)), dtype=np.uint32) for _ in range(40)]
    ids = [server.submit_sumcheck(t) for t in tables]
    res = _wait(server, ids)
    server.close()
    for t, i in zip(tables, ids):
        want = oracle.sumcheck_multilinear(t)
        got = res[i][0]
        assert got["claimed_sum"] == want["claimed_sum"] and got["final"] == want["final"]
        assert got["initial_digest"] == want["initial_digest"]
        for key in ("r0", "r1", "challenges"):
            assert np.array_equal(got[key], want[key])


def test_nocopy_submissions_match_copied(ctx, oracle):
    """Jobs submitted without a copy (the server reads the caller's arrays when a
    worker takes them) give the bytes of the copied submissions; the wrapper holds
    each array until the job is seen finished, and a non-canonical word is still
    refused at submission."""
    rng = np.random.default_rng(0x0C0)
    server = azk.ProofServer(ctx, hbm_budget_bytes=4 << 30, slots=4)
    jobs = [_pcs_job(rng, int(k)) for k in rng.integers(10, 17, 16)]
    tables = [rng.integers(0, P, 1 << int(k), dtype=np.uint32) for k in rng.integers(8, 16, 8)]
    ids = [server.submit_pcs(j["log_size"], 2, j["queries"], j["rounds"], j["coeffs"], j["pub"], copy=False) for j in jobs]
    sids = [server.submit_sumcheck(t, copy=False) for t in tables]
    with pytest.raises(azk.AZKError) as e:
        server.submit_sumcheck(np.full(16, P, np.uint32), copy=False)
    assert e.value.name == "invalidInputLayout"
    res = _wait(server, ids + sids)
    assert not server._borrowed
    cids = [server.submit_pcs(j["log_size"], 2, j["queries"], j["rounds"], j["coeffs"], j["pub"]) for j in jobs]
    csids = [server.submit_sumcheck(t) for t in tables]
    cres = _wait(server, cids + csids)
    server.close()
    for a, b in zip(ids, cids):
        assert res[a][0] == cres[b][0]
    for t, a, b in zip(tables, sids, csids):
        want = oracle.sumcheck_multilinear(t)
        for got in (res[a][0], cres[b][0]):
            assert got["initial_digest"] == want["initial_digest"] and got["final"] == want["final"]
            assert np.array_equal(got["challenges"], want["challenges"])


def test_lane_smallest_tables_beside_larger_ones(ctx, oracle):
    """Tables of 2, 4 and 8 evaluations (the round-0 sums of the smallest taken by
    one thread, the fold of the last rounds by one thread) share packed launches
    with larger tables and each give the oracle's proof."""
    rng = np.random.default_rng(0x5C6)
    server = azk.ProofServer(ctx, hbm_budget_bytes=1 << 30, slots=2)
    sizes = [1, 2, 3, 12, 1, 9, 2, 16, 3, 1, 5]
    tables = [rng.integers(0, P, 1 << k, dtype=np.uint32) for k in sizes]
    ids = [server.submit_sumcheck(t, copy=False) for t in tables]
    res = _wait(server, ids)
    server.close()
    for t, i in zip(tables, ids):
        want = oracle.sumcheck_multilinear(t)
        got = res[i][0]
        assert got["claimed_sum"] == want["claimed_sum"] and got["final"] == want["final"]
        assert got["initial_digest"] == want["initial_digest"]
        for key in ("r0", "r1", "challenges"):
            assert np.array_equal(got[key], want[key])
