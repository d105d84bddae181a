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
