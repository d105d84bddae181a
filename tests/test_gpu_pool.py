"""The job pool on the GPU: each job's result is the same alone and in the mix, and
admission keeps the running jobs inside the memory budget while queued jobs enter as
others finish (continuous batching).

Tolerances: deterministic mode (fixed-point deposit) must be bit-identical alone and in
the mix; fast mode (float atomics in scheduling order) within the 100-step trajectory bar
of the parity tests scaled to these 20 steps: max |dx| <= 1e-3, median <= 1e-5.
"""
import numpy as np
import pytest

import tild_b200
from tild_b200 import synth

pytestmark = pytest.mark.gpu

SPECS = {
    "diblock_o3": lambda: synth.small_system(seed=51, order=3),
    "charged_o4": lambda: synth.small_system(seed=52, order=4, charges=True, n_free=30),
    "erf_o2": lambda: synth.small_system(seed=53, order=2, grid=(15, 12, 18), pots=[
        dict(kind="erf2", I="A", J="B", A=0.05, Rp=1.0, sigma=0.5),
        dict(kind="gaussian", I="all", J="all", A=1.0, sigma=0.7)]),
    "bigger_o3": lambda: synth.small_system(seed=54, order=3, n_chains=200, nper=10, L=12.0, grid=(24, 24, 24),
                                            charges=True),
}
NSTEPS = 20
# a job whose 96^3 grid needs several times the memory of the small systems above
BIG = lambda: synth.small_system(seed=55, order=3, n_chains=40, L=20.0, grid=(96, 96, 96))  # noqa: E731


def alone(spec, **opts):
    o = {"write_files": 0, "sort_interval": 3}
    o.update(opts)
    with tild_b200.box_from_spec(spec, options=o) as b:
        b.command("endBox")
        b.step(NSTEPS)
        return b.positions(), np.asarray(b.thermo_raw())


def in_mix(specs, budget=8 << 30, max_active=0, **opts):
    o = {"write_files": 0, "sort_interval": 3}
    o.update(opts)
    out = {}
    with tild_b200.Pool(mem_budget_bytes=budget, max_active=max_active) as pool:
        ids = {}
        for name, spec in specs.items():
            b = tild_b200.box_from_spec(spec, options=o)
            ids[name] = (pool.submit(b, NSTEPS), spec.N)
            b.close()
        for name, (jid, n) in ids.items():
            pool.wait(jid)
            x, th = pool.result(jid, n)
            out[name] = (x, th, pool.status(jid))
        assert pool.stats()["done"] == len(specs) and pool.stats()["bytes_in_use"] == 0
    return out


def test_deterministic_results_identical_alone_and_in_the_mix():
    specs = {k: f() for k, f in SPECS.items()}
    mix = in_mix(specs, deterministic=1)
    for name, spec in specs.items():
        xa, tha = alone(spec, deterministic=1)
        xm, thm, st = mix[name]
        assert st["state"] == "done" and st["steps_done"] == NSTEPS
        assert np.array_equal(xa, xm), name
        assert np.array_equal(tha[: len(thm)], thm), name


def test_fast_mode_results_match_alone_within_tolerance():
    specs = {k: f() for k, f in SPECS.items()}
    mix = in_mix(specs)
    for name, spec in specs.items():
        xa, _ = alone(spec)
        xm = mix[name][0]
        d = np.abs(xa - xm)
        d = np.minimum(d, np.asarray(spec.L, np.float32) - d)
        assert d.max() <= 1e-3 and np.median(d) <= 1e-5, (name, d.max(), np.median(d))


def test_admission_respects_max_active_and_refills():
    base = SPECS["diblock_o3"]
    specs = {"j%d" % i: synth.small_system(seed=60 + i, order=3) for i in range(6)}
    mix = in_mix(specs, max_active=2, deterministic=1)
    spans = sorted((r[2]["admit_s"], r[2]["done_s"]) for r in mix.values())
    for a, _ in spans:   # never more than two jobs running at once
        assert sum(1 for a2, d2 in spans if a2 <= a < d2) <= 2
    # the third job entered only after one of the first two had finished
    first_done = min(d for _, d in spans[:2])
    assert spans[2][0] >= first_done
    for name, spec in specs.items():
        xa, _ = alone(spec, deterministic=1)
        assert np.array_equal(xa, mix[name][0]), name
    assert base is not None


def test_pool_refuses_a_job_larger_than_its_budget():
    with tild_b200.Pool(mem_budget_bytes=2 << 20) as pool:
        b = tild_b200.box_from_spec(SPECS["bigger_o3"](), options={"write_files": 0})
        with pytest.raises(tild_b200.TildError, match="budget"):
            pool.submit(b, 5)
        b.command("endBox")   # the caller still owns a usable box
        b.step(2)
        assert np.isfinite(b.positions()).all()
        b.close()


def _submit(pool, spec, nsteps, **opts):
    o = {"write_files": 0, "sort_interval": 3, "deterministic": 1}
    o.update(opts)
    b = tild_b200.box_from_spec(spec, options=o)
    jid = pool.submit(b, nsteps)
    b.close()
    return jid


def _wait_until(pred, timeout=60.0):
    import time
    t0 = time.time()
    while not pred():
        assert time.time() - t0 < timeout, "condition not reached"
        time.sleep(0.005)


def test_cancel_a_running_job_frees_it_and_leaves_the_others_alone():
    spec = SPECS["diblock_o3"]()
    other = SPECS["charged_o4"]()
    with tild_b200.Pool(mem_budget_bytes=8 << 30) as pool:
        long_job = _submit(pool, spec, 10 ** 7)          # would run for minutes
        keep = _submit(pool, other, NSTEPS)
        _wait_until(lambda: pool.status(long_job)["steps_done"] > 0)
        pool.cancel(long_job)
        with pytest.raises(tild_b200.TildError, match="cancelled"):
            pool.wait(long_job)
        st = pool.status(long_job)
        assert st["state"] == "cancelled" and 0 < st["steps_done"] < 10 ** 7
        with pytest.raises(tild_b200.TildError, match="already finished"):
            pool.cancel(long_job)
        pool.wait(keep)
        x, th = pool.result(keep, other.N)
        s = pool.stats()
        assert s["cancelled"] == 1 and s["done"] == 1 and s["bytes_in_use"] == 0 and s["running"] == 0
        pool.release(long_job)
    xa, tha = alone(other, deterministic=1)
    assert np.array_equal(xa, x) and np.array_equal(tha[: len(th)], th)


def test_cancel_a_queued_job():
    with tild_b200.Pool(mem_budget_bytes=8 << 30, max_active=1) as pool:
        running = _submit(pool, SPECS["diblock_o3"](), 10 ** 7)
        queued = _submit(pool, SPECS["erf_o2"](), NSTEPS)
        _wait_until(lambda: pool.status(running)["state"] == "running")
        assert pool.status(queued)["state"] == "queued"
        pool.cancel(queued)
        st = pool.status(queued)
        assert st["state"] == "cancelled" and st["steps_done"] == 0 and st["admit_s"] == 0.0
        pool.cancel(running)
        with pytest.raises(tild_b200.TildError, match="cancelled"):
            pool.wait(running)
        assert pool.stats()["cancelled"] == 2 and pool.stats()["bytes_in_use"] == 0


def test_a_stalled_producer_does_not_hold_back_running_jobs():
    """Jobs submitted with long pauses between them: the first runs to completion while
    the producer is stalled, and each result equals the job run alone."""
    import time
    specs = [SPECS["diblock_o3"](), SPECS["charged_o4"]()]
    with tild_b200.Pool(mem_budget_bytes=8 << 30) as pool:
        first = _submit(pool, specs[0], NSTEPS)
        _wait_until(lambda: pool.status(first)["state"] == "done")   # no further submit meanwhile
        time.sleep(0.2)
        second = _submit(pool, specs[1], NSTEPS)
        pool.wait(second)
        s1, s2 = pool.status(first), pool.status(second)
        assert s1["done_s"] < s2["submit_s"]
        for jid, spec in ((first, specs[0]), (second, specs[1])):
            x, _ = pool.result(jid, spec.N)
            assert np.array_equal(x, alone(spec, deterministic=1)[0])


def test_budget_lowered_below_the_running_set():
    """Running jobs keep their memory and finish; a queued job enters only once the
    running set fits the new budget; a queued job larger than the new budget fails."""
    spec = SPECS["diblock_o3"]()
    with tild_b200.Pool(mem_budget_bytes=8 << 30) as pool:
        a = _submit(pool, spec, 20000)   # long enough to still run when the budget drops
        b = _submit(pool, spec, 20000)
        _wait_until(lambda: pool.stats()["running"] == 2)
        per_job = pool.stats()["bytes_in_use"] // 2
        pool.set_budget(per_job + per_job // 2)   # below the two running jobs
        c = _submit(pool, spec, NSTEPS)
        assert pool.status(c)["state"] == "queued"
        pool.wait(a)
        pool.wait(b)
        pool.wait(c)
        sa, sb, sc = pool.status(a), pool.status(b), pool.status(c)
        assert sa["steps_done"] == sb["steps_done"] == 20000 and sc["steps_done"] == NSTEPS
        assert sc["admit_s"] >= min(sa["done_s"], sb["done_s"])   # entered after one had left
        with pytest.raises(tild_b200.TildError, match="budget"):
            pool.submit(tild_b200.box_from_spec(BIG(), options={"write_files": 0}), 5)
    with tild_b200.Pool(mem_budget_bytes=8 << 30, max_active=1) as pool:
        r = _submit(pool, spec, 10 ** 7)
        q = _submit(pool, BIG(), NSTEPS)
        _wait_until(lambda: pool.status(r)["state"] == "running")
        pool.set_budget(pool.stats()["bytes_in_use"])   # the running job still fits; the queued one cannot
        st = pool.status(q)
        assert st["state"] == "failed"
        with pytest.raises(tild_b200.TildError, match="budget"):
            pool.wait(q)
        pool.cancel(r)
        with pytest.raises(tild_b200.TildError, match="cancelled"):
            pool.wait(r)
