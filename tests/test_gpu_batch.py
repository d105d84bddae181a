"""Batched replicas (tild_batch_*): every stage of a step is one launch over all replicas.

A batch must give each replica exactly the trajectory it has when stepped alone: in
deterministic mode (64-bit fixed-point deposit) the positions after steps with a re-sort
in between are bit-identical.  Boxes the batch's shared kernels cannot serve are refused
with a reason."""
import ctypes

import numpy as np
import pytest

import tild_b200
from tild_b200 import synth

pytestmark = pytest.mark.gpu


def replicas():
    """Three uneven diblock-like systems: different sizes, grids (one with a prime edge),
    box lengths, amplitudes and seeds."""
    specs = [
        synth.small_system(seed=41, n_chains=60, nper=10, L=8.0, grid=(16, 16, 16)),
        synth.small_system(seed=42, n_chains=150, nper=8, L=10.0, grid=(20, 20, 24)),
        synth.small_system(seed=43, n_chains=90, nper=12, L=9.0, grid=(17, 18, 18), pots=[
            dict(kind="gaussian", I="A", J="A", A=1.5, sigma=0.7),
            dict(kind="gaussian", I="A", J="B", A=4.0, sigma=0.7),
            dict(kind="gaussian", I="B", J="B", A=1.5, sigma=0.7)]),
    ]
    return specs


def make(spec, **opts):
    o = {"write_files": 0}
    o.update(opts)
    b = tild_b200.box_from_spec(spec, options=o)
    b.command("endBox")
    return b


@pytest.mark.parametrize("order,streams", [(2, 1), (3, 1), (3, 2)])
def test_batch_matches_replicas_stepped_alone(order, streams):
    specs = replicas()
    for s in specs:
        s.order = order
    steps = 23   # re-sorts at steps 10 and 20 (sort_interval 10)
    alone = []
    for s in specs:
        with make(s, deterministic=1) as b:
            b.step(steps)
            alone.append(b.positions())
    boxes = [make(s, deterministic=1) for s in specs]
    with tild_b200.Batch(streams=streams) as batch:
        for b in boxes:
            batch.add(b)
        assert len(batch) == len(specs)
        batch.step(7)
        batch.step(steps - 7)
    for b, x in zip(boxes, alone):
        assert b.info().step == steps
        assert np.array_equal(b.positions(), x)
        b.close()


def test_batch_fast_mode_matches_within_trajectory_tolerance():
    """Fast mode (int32 tile boxes, FP32 flush atomics): the same kernels, sums in another
    order; 20 steps agree to the trajectory tolerance of the parity suite."""
    specs = replicas()
    alone = []
    for s in specs:
        with make(s) as b:
            b.step(20)
            alone.append(b.positions())
    boxes = [make(s) for s in specs]
    with tild_b200.Batch() as batch:
        for b in boxes:
            batch.add(b)
        batch.step(20)
    for b, x, s in zip(boxes, alone, specs):
        d = b.positions() - x
        d -= np.round(d / s.L[:3]) * s.L[:3]
        assert np.abs(d).max() <= 1e-3 and np.median(np.abs(d)) <= 1e-4
        b.close()


def test_batch_refuses_what_it_cannot_serve():
    specs = replicas()
    ok = make(specs[0])
    charged = make(synth.small_system(seed=44, order=3, charges=True))   # three density fields
    other_order = make(synth.small_system(seed=45, order=2))
    not_ready = tild_b200.box_from_spec(specs[1], options={"write_files": 0})
    with tild_b200.Batch() as batch:
        batch.add(ok)
        for b, code in ((charged, "UNSUPPORTED"), (other_order, "UNSUPPORTED"), (not_ready, "STATE")):
            with pytest.raises(tild_b200.TildError, match=code):
                batch.add(b)
        with pytest.raises(tild_b200.TildError, match="STATE"):
            batch.add(ok)   # already a member
        # a member cannot be destroyed while the batch lives
        rc = tild_b200.lib().tild_box_destroy(ok._h)
        assert rc != tild_b200.TILD_OK and "batch" in tild_b200.lib().tild_last_error().decode()
        assert len(batch) == 1
    for b in (ok, charged, other_order, not_ready):
        b.close()


def test_batch_c3_like_replicas_run():
    """A few replicas drawn like the C3 workload (N log-uniform, grids at spacing 0.4,
    chain lengths 16..48) step through the batch and stay finite and inside their boxes."""
    specs = synth.config_c3(replicas=4, seed=7, nmax=4.0e4)
    boxes = [make(s) for s in specs]
    with tild_b200.Batch() as batch:
        for b in boxes:
            batch.add(b)
        batch.step(30)
    for b, s in zip(boxes, specs):
        x = b.positions()
        assert np.isfinite(x).all() and (x >= 0).all() and (x <= s.L[:3]).all()
        b.close()


ANGLES = [dict(style="harmonic", k=3.0, theta=120.0), dict(style="wlc", k=2.0)]


@pytest.mark.parametrize("kind", ["one_force_group", "angles", "curand_noise", "em"])
def test_batch_other_kernel_settings_match_alone(kind):
    """The batch's other instantiations: one density field and force group (a homopolymer
    with one Gaussian), replicas with angles (the integrator pass's extra terms), the
    cuRAND-compatible noise (per-particle generator states) and the EM integrator; each
    replica bit-identical in deterministic mode to its run alone."""
    opts = {"deterministic": 1}
    if kind == "one_force_group":
        pots = [dict(kind="gaussian", I="all", J="all", A=3.0, sigma=0.7)]
        specs = [synth.small_system(seed=50 + k, n_chains=70 + 30 * k, nper=8, L=8.0 + k, grid=(16 + 2 * k,) * 3,
                                    pots=pots) for k in range(3)]
    elif kind == "angles":
        specs = [synth.small_system(seed=60 + k, n_chains=60 + 20 * k, nper=10, L=8.0, grid=(16, 16, 18),
                                    angle_params=ANGLES) for k in range(2)]
    elif kind == "curand_noise":
        specs = replicas()
        opts["rng"] = 1
    else:
        specs = [synth.small_system(seed=70 + k, n_chains=80, nper=8, L=8.0, grid=(16, 16, 16), integrator="EM")
                 for k in range(2)]
    alone = []
    for s in specs:
        with make(s, **opts) as b:
            b.step(12)
            alone.append(b.positions())
    boxes = [make(s, **opts) for s in specs]
    with tild_b200.Batch() as batch:
        for b in boxes:
            batch.add(b)
        batch.step(12)
    for b, x in zip(boxes, alone):
        assert np.array_equal(b.positions(), x)
        b.close()
