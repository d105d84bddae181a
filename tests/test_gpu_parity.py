"""GPU parity of the CUDA TILD path against the CPU oracle, through the C ABI.

Tolerances (written here, used below):
  * stencil indices: bit-exact with the FP32 restatement of d_calcGridWeights;
    weights: bit-exact as well (same IEEE operations, explicit FMAs);
  * densities: |drho| <= 1e-6 * max|rho| (FP32 atomics vs FP64 sums);
  * forces: max_p |df_p| / max(|f_p|, f_rms) <= 1e-5 against the FP64 oracle, raised by
    2^-21/sin^2(theta) for the particles of a near-straight angle (FP32 conditioning);
  * energies: relative 1e-5 (pair terms) and 1e-6 (bond term);
  * 100-step GJF trajectories with identical Philox noise: max |dx| <= 2e-4.
"""
import os

import numpy as np
import pytest

import oracle
import tild_b200
from conftest import angle_force_tolerance, force_error, spec_to_system
from tild_b200 import synth

pytestmark = pytest.mark.gpu

F_TOL = 1e-5
ANGLES = [dict(style="harmonic", k=3.0, theta=120.0), dict(style="wlc", k=2.0)]


def make_box(spec, **opts):
    o = {"write_files": 0}
    o.update(opts)
    b = tild_b200.box_from_spec(spec, options=o)
    b.command("endBox")
    return b


SYSTEMS = {
    "diblock_o3": lambda: synth.small_system(seed=1, order=3),
    "charged_o3": lambda: synth.small_system(seed=2, order=3, charges=True),
    "o0": lambda: synth.small_system(seed=3, order=0),
    "o1": lambda: synth.small_system(seed=4, order=1),
    "o2": lambda: synth.small_system(seed=5, order=2),
    "o4_quirk": lambda: synth.small_system(seed=6, order=4),
    "erf": lambda: synth.small_system(seed=7, order=3, pots=[
        dict(kind="erf2", I="A", J="B", A=0.05, Rp=1.0, sigma=0.5),
        dict(kind="erfG", I="B", J="B", A=0.3, Rp=0.8, sigma=0.5),
        dict(kind="gaussian", I="all", J="A", A=1.5, sigma=0.8)]),
    "odd_grid": lambda: synth.small_system(seed=8, order=3, grid=(15, 9, 21), charges=True),
    # odd x with an odd number of lines per x-inverse block (45: 3 pairs x 19 lines)
    "odd_grid_wide": lambda: synth.small_system(seed=10, order=3, grid=(45, 10, 12), L=9.0, charges=True),
    # radix-7 stages on every axis, and generic prime radices 11 and 13
    "radix7_grid": lambda: synth.small_system(seed=12, order=2, grid=(21, 14, 28), L=7.0, charges=True),
    "prime_grid": lambda: synth.small_system(seed=13, order=1, grid=(22, 13, 11), charges=True),
    # whole prime lines (one generic butterfly of radix n per line) on every axis
    "prime_lines": lambda: synth.small_system(seed=14, order=3, grid=(31, 37, 29), L=11.0, charges=True),
    "angles": lambda: synth.small_system(seed=15, order=3, charges=True, angle_params=ANGLES),
    "free_particles": lambda: synth.small_system(seed=9, order=3, n_free=50, charges=True),
    # combs (degree 3) and stars (degree 5): rows of every length in the CSR bond list
    "branched": lambda: synth.branched_system(seed=3),
    # harmonic walls (per-particle potentials) beside grid potentials
    "walls": lambda: synth.small_system(seed=22, order=3, charges=True, pots=[
        dict(kind="gaussian", I="A", J="B", A=2.0, sigma=0.7), dict(kind="charges", lB=1.0, sigma=0.5),
        dict(kind="wall", I="A", axis="z", pos=2.0, sign=1, k=5.0),
        dict(kind="wall", I="all", axis="x", pos=4.5, sign=-1, k=3.0)]),
    # 2-D boxes: one grid plane, particles at z = 0
    "d2_charged": lambda: synth.small_system(seed=20, order=3, charges=True, dim=2, grid=(16, 18, 1)),
    "d2_o4_angles": lambda: synth.small_system(seed=21, order=4, dim=2, grid=(15, 12, 1), angle_params=ANGLES),
}


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_forces_match_oracle(name):
    spec = SYSTEMS[name]()
    sysm = spec_to_system(spec)
    with make_box(spec) as b:
        f = b.forces()
    fref, _ = oracle.forces(sysm, prec=64)
    err = force_error(f, fref, angle_force_tolerance(sysm, F_TOL))
    assert err <= 1.0, "%s: force error %.3g of the tolerance" % (name, err)


@pytest.mark.parametrize("name", ["charged_o3", "erf", "odd_grid", "prime_lines", "radix7_grid"])
def test_grid_forces_match_oracle(name):
    """The spectral stage alone (cufftWrapperSingle + CalcForces, Box.cu:107-127,
    ps_potential.cu:41-125): every force group's grid force (PS_Group::d_gridForce) after
    a force evaluation against the oracle's FP64 transforms of the FP64 densities, within
    1e-5 of the field's largest value, and zeros for a group without grid force."""
    spec = SYSTEMS[name]()
    sysm = spec_to_system(spec)
    _, inter = oracle.forces(sysm, prec=64)
    glist = oracle.groups(sysm)
    with make_box(spec) as b:
        b.forces()
        for gi, (gname, _, _) in enumerate(glist):
            gf = b.grid_force(gname)
            if gi not in inter["gridforce"]:
                assert not gf.any(), gname
                continue
            ref = inter["gridforce"][gi].T
            assert np.abs(gf - ref).max() <= 1e-5 * np.abs(ref).max(), gname


@pytest.mark.parametrize("order", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("exact4", [0, 1])
def test_grid_weights_bit_exact(order, exact4):
    if exact4 and order != 4:
        pytest.skip("exact flag only changes order 4")
    spec = synth.small_system(seed=20 + order, order=order)
    rng = np.random.default_rng(order)
    # edge cases: 0, exactly on grid lines/cell centres, just below L, exactly L
    L = spec.L
    h = L / spec.grid
    extra = np.array([[0, 0, 0], L * 0.999999, L, h * 3, h * 3.5, h * 2.5 + 1e-6], np.float32)
    spec.x = np.concatenate([spec.x, extra]).astype(np.float32)
    spec.types = np.r_[spec.types, np.zeros(len(extra), np.int32)]
    spec.mol = np.r_[spec.mol, np.arange(len(extra)) + 10000].astype(np.int32)
    sysm = spec_to_system(spec, quirk4=0 if exact4 else 1)
    with make_box(spec, bspline4_exact=exact4) as b:
        inds, w = b.grid_weights()
    ri, rw = oracle.weights(sysm, prec=32)
    assert np.array_equal(inds, ri)
    assert np.array_equal(w.view(np.uint32), rw.astype(np.float32).view(np.uint32))


def test_densities_match_oracle():
    spec = synth.small_system(seed=11, order=3, charges=True)
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm, prec=64)
    with make_box(spec) as b:
        for name, (rho, rhoq) in dens.items():
            got = b.density(name)
            assert np.abs(got - rho).max() <= 1e-6 * np.abs(rho).max()
            if rhoq is not None:
                gq = b.density(name, charge=True)
                assert np.abs(gq - rhoq).max() <= 1e-6 * np.abs(rhoq).max()


@pytest.mark.parametrize("name", ["diblock_o3", "charged_o3", "erf", "odd_grid", "prime_lines", "walls", "branched"])
def test_energies_match_oracle(name):
    spec = SYSTEMS[name]()
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm)
    ref = oracle.pair_energies(sysm, dens)
    ub, vir = oracle.bond_energy(sysm)
    with make_box(spec) as b:
        t = b.thermo()
    for e, r in zip(t["potentials"], ref):
        assert abs(e - r) <= 1e-5 * max(abs(r), 1e-12) + 1e-9, (e, r)
    assert abs(t["Ubond"] - ub) <= 1e-6 * abs(ub)
    assert abs(t["Upe"] - (sum(ref) + ub)) <= 1e-5 * abs(sum(ref) + ub)


def test_deterministic_mode_bit_reproducible_and_accurate():
    spec = synth.small_system(seed=12, order=3, charges=True)
    sysm = spec_to_system(spec)
    fref, _ = oracle.forces(sysm)
    outs = []
    for _ in range(2):
        with make_box(spec, deterministic=1) as b:
            outs.append(b.forces())
            b.step(5)
            outs.append(b.positions())
    assert np.array_equal(outs[0], outs[2]) and np.array_equal(outs[1], outs[3])
    assert force_error(outs[0], fref) <= F_TOL


def test_autotuned_tiles_are_invisible():
    """The tile autotuner only changes the work split: in deterministic mode the forces and
    a short trajectory are bit-identical with and without it."""
    spec = synth.small_system(seed=26, order=3, charges=True, n_chains=120, nper=10, L=10.0, grid=(20, 20, 20))
    outs = []
    for tune in (0, 1):
        with make_box(spec, deterministic=1, autotune=tune) as b:
            outs.append((b.forces(), b.describe()["tiles"]))
            b.step(5)
            outs[-1] += (b.positions(),)
    assert outs[1][1]["autotuned"] and outs[1][1]["tuned_ms"] > 0
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][2], outs[1][2])


@pytest.mark.parametrize("order", [2, 3, 4])
def test_deposit_tiles_are_invisible(order):
    """The deposit's own tile size (bricks per CTA) only changes the work split: in
    deterministic mode the forces and a short trajectory are bit-identical for every size."""
    spec = synth.small_system(seed=28, order=order, charges=True, n_chains=120, nper=10, L=10.0, grid=(20, 20, 20))
    outs = []
    for codes in (8, 16, 32, 64):
        with make_box(spec, deterministic=1, deposit_codes=codes) as b:
            assert b.describe()["tiles"]["deposit_codes"] == codes
            f = b.forces()
            b.step(5)
            outs.append((f, b.positions()))
    for f, x in outs[1:]:
        assert np.array_equal(outs[0][0], f) and np.array_equal(outs[0][1], x)


@pytest.mark.parametrize("qscale", [1.0, 0.5])
@pytest.mark.parametrize("codes", [8, 32])
def test_forces_and_energies_match_oracle_deposit_tiles(qscale, codes):
    """Fast-mode forces and pair energies against the FP64 oracle for small and large
    deposit tiles, with charges of +-1 (one fixed-point conversion per stencil point serves
    every density field) and of +-0.5 (a conversion per field)."""
    spec = synth.small_system(seed=29, order=3, charges=True, n_chains=120, nper=10, L=10.0, grid=(20, 20, 20))
    spec.charges = (spec.charges * qscale).astype(np.float32)
    sysm = spec_to_system(spec)
    fref, _ = oracle.forces(sysm, prec=64)
    dens, _, _ = oracle.densities(sysm)
    ref = oracle.pair_energies(sysm, dens)
    with make_box(spec, deposit_codes=codes) as b:
        f = b.forces()
        t = b.thermo()
    assert force_error(f, fref) <= 1e-5
    for e, r in zip(t["potentials"], ref):
        assert abs(e - r) <= 1e-5 * max(abs(r), 1e-12) + 1e-9, (e, r)


@pytest.mark.parametrize("n_chains", [120, 300])
def test_large_deposit_tiles_match_oracle(n_chains):
    """Deposit tiles of 64 bricks on a dense coacervate-like system: their particle counts
    exceed the int32 box's count bound at 2^24 per unit weight, so the box sums at 2^23 or
    2^22 (or in FP32 beyond); forces and energies against the FP64 oracle stay within 1e-5."""
    pots = [dict(kind="gaussian", I="all", J="all", A=2.0, sigma=0.7), dict(kind="charges", lB=1.0, sigma=0.5)]
    spec = synth.small_system(seed=31, order=3, charges=True, n_chains=n_chains, nper=10, L=10.0, grid=(20, 20, 20),
                              pots=pots)
    sysm = spec_to_system(spec)
    fref, _ = oracle.forces(sysm, prec=64)
    dens, _, _ = oracle.densities(sysm)
    ref = oracle.pair_energies(sysm, dens)
    with make_box(spec, deposit_codes=64) as b:
        f = b.forces()
        t = b.thermo()
    assert force_error(f, fref) <= 1e-5
    for e, r in zip(t["potentials"], ref):
        assert abs(e - r) <= 1e-5 * max(abs(r), 1e-12) + 1e-9, (e, r)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_direct_gather_is_invisible(order):
    """Reading every stencil through L1/L2 instead of the tile's staged box changes only
    where the records come from: forces and a short trajectory are bit-identical."""
    spec = synth.small_system(seed=27, order=order, charges=True, n_chains=120, nper=10, L=10.0, grid=(20, 20, 20))
    outs = []
    for direct in (0, 1):
        with make_box(spec, deterministic=1, direct_gather=direct) as b:
            outs.append((b.forces(), b.describe()["tiles"]["gather"]))
            b.step(5)
            outs[-1] += (b.positions(),)
    assert [o[1] for o in outs] == ["staged", "direct"]
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][2], outs[1][2])


def test_blown_up_positions_are_reported_as_err_device():
    """A position that is NaN or infinite (a run that blew up) is counted on the device and
    reported as ERR_DEVICE when the energies are read, instead of logging NaN; the box
    stays usable once the positions are finite again.  Every index stays on the grid for
    such positions: stencil origins and sort cells are wrapped or clamped."""
    spec = synth.small_system(seed=31, order=3, charges=True, n_chains=40, nper=10, L=10.0, grid=(20, 20, 20))
    with make_box(spec) as b:
        x = b.positions()
        ok = b.thermo()
        for bad in (np.nan, np.inf):
            y = x.copy()
            y[7, 1] = bad
            y[123, 2] = bad
            b.set_positions(y)
            with pytest.raises(tild_b200.TildError) as ei:
                b.thermo()
            assert ei.value.code == 7 and "2 particle(s) with a non-finite position" in str(ei.value)
        b.set_positions(x)
        again = b.thermo()
        assert np.allclose(again["potentials"], ok["potentials"], rtol=1e-6)


def test_spatial_sort_is_invisible_tile_gather():
    """The same for a box of two force groups, whose sorted steps take the tile gather over
    paired records and whose unsorted ones (sort_interval 0) the planar gather."""
    spec = synth.small_system(seed=19, order=3, n_free=30)
    outs = []
    for interval in (0, 3, 1):
        with make_box(spec, deterministic=1, sort_interval=interval) as b:
            f = b.forces()
            b.step(10)
            outs.append((f, b.positions(), b.forces()))
    for o in outs[1:]:
        for a, b2 in zip(outs[0], o):
            assert np.array_equal(a, b2)


@pytest.mark.parametrize("order", [2, 3])
def test_gather_threads_are_invisible(order):
    """The tile gather's CTA size (option gather_threads) decides how a tile's particles
    are spread over warps and passes, not what a particle's sum is: forces and a trajectory
    with re-sorts are bit-identical from 64 to 448 threads (tiles of 1 and 4 bricks on a
    scaled coacervate, so that passes hold both full and ragged warps)."""
    spec = synth.config_c2(scale=0.03)
    spec.order = order
    for codes in (1, 4):
        outs = []
        for thr in (0, 64, 160, 448):
            with make_box(spec, deterministic=1, tile_codes=codes, gather_threads=thr) as b:
                f = b.forces()
                b.step(12)
                outs.append((f, b.positions(), b.forces()))
        for o in outs[1:]:
            for a, b2 in zip(outs[0], o):
                assert np.array_equal(a, b2)


def test_spatial_sort_is_invisible():
    """Re-sorting the particle arrays changes only memory order: in deterministic mode the
    trajectory is bit-identical with no sort, a sort every 3 steps and every step."""
    spec = synth.small_system(seed=18, order=3, charges=True, n_free=30)
    outs = []
    for interval in (0, 3, 1):
        with make_box(spec, deterministic=1, sort_interval=interval) as b:
            f = b.forces()
            b.step(10)
            outs.append((f, b.positions(), b.forces()))
    for o in outs[1:]:
        for a, r in zip(o, outs[0]):
            assert np.array_equal(a, r)


def test_branched_bonds_sorted_and_integrated_like_the_oracle():
    """The CSR bond list under re-sorting: combs and stars (rows of 0 to 5 partners) keep
    bit-identical trajectories with no sort and a sort every step (deterministic mode),
    their bond energy matches the oracle after the steps, and 100 Philox steps follow the
    FP64 oracle fed the same noise (the drift bar of the linear chains)."""
    spec = synth.branched_system(seed=4)
    outs = []
    for interval in (0, 1):
        with make_box(spec, deterministic=1, sort_interval=interval) as b:
            b.step(20)
            outs.append((b.positions(), b.forces(), b.thermo()["Ubond"]))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]
    sysm = spec_to_system(spec)
    sysm.x = outs[0][0].astype(np.float32)
    ub, _ = oracle.bond_energy(sysm)
    assert abs(outs[0][2] - ub) <= 1e-6 * abs(ub)
    sysm = spec_to_system(spec)
    traj = oracle.Trajectory(sysm, 64)
    ids = np.arange(sysm.N)
    with make_box(spec, sort_interval=1) as b:
        b.step(100)
        x = b.positions()
    for step in range(100):
        traj.step(oracle.philox_normals(spec.seed, step, ids))
    d = np.abs(x - traj.positions())
    d = np.minimum(d, spec.L - d)
    assert d.max() <= 1e-3 and np.median(d) <= 1e-4, (d.max(), np.median(d))


@pytest.mark.parametrize("integ", ["GJF", "EM"])
def test_trajectory_matches_oracle_100_steps(integ):
    spec = synth.small_system(seed=13, order=3, charges=True)
    spec.integrator = integ
    sysm = spec_to_system(spec)
    traj = oracle.Trajectory(sysm, 64)
    ids = np.arange(sysm.N)
    with make_box(spec) as b:
        b.step(100)
        x = b.positions()
    for step in range(100):
        traj.step(oracle.philox_normals(spec.seed, step, ids))
    d = np.abs(x - traj.positions())
    d = np.minimum(d, spec.L - d)
    # stated drift: the FP32 restatement itself drifts 4.7e-4 (max) from FP64 here
    assert d.max() <= 1e-3 and np.median(d) <= 1e-4, (d.max(), np.median(d))


def test_tiles_without_grid_forces_integrate_like_the_oracle():
    """Species B takes no grid force and fills half of the box, so whole tiles gather
    nothing: their particles still integrate with their own x_{t-1}, noise and id."""
    spec = synth.small_system(seed=19, order=3, n_chains=40, nper=8,
                              pots=[dict(kind="gaussian", I="A", J="A", A=2.0, sigma=0.7)])
    spec.types = (spec.x[:, 0] >= spec.L[0] / 2).astype(np.int32)
    sysm = spec_to_system(spec)
    traj = oracle.Trajectory(sysm, 64)
    ids = np.arange(sysm.N)
    with make_box(spec, sort_interval=5) as b:
        b.step(30)
        x = b.positions()
    for step in range(30):
        traj.step(oracle.philox_normals(spec.seed, step, ids))
    d = np.abs(x - traj.positions())
    d = np.minimum(d, spec.L - d)
    assert d.max() <= 1e-3 and np.median(d) <= 1e-4, (d.max(), np.median(d))


@pytest.mark.parametrize("name", ["d2_charged", "d2_o4_angles"])
def test_2d_trajectory_energies_and_pressure_match_oracle(name):
    spec = SYSTEMS[name]()
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm)
    ref = oracle.pair_energies(sysm, dens)
    with make_box(spec) as b:
        th = b.thermo()
        for k, r in enumerate(ref):
            assert abs(th["potentials"][k] - r) <= 1e-5 * max(abs(r), 1e-9)
        assert th["pressure"][2] == 0.0   # zz: no kinetic or virial term in a plane
        b.step(50)
        x = b.positions()
    assert x.shape == (spec.N, 2)
    traj = oracle.Trajectory(sysm, 64)
    ids = np.arange(sysm.N)
    for step in range(50):
        traj.step(oracle.philox_normals(spec.seed, step, ids))
    d = np.abs(x - traj.positions())
    d = np.minimum(d, np.asarray(spec.L[:2]) - d)
    assert d.max() <= 1e-3 and np.median(d) <= 1e-4, (d.max(), np.median(d))


def test_forces_unchanged_by_forces_call_and_positions_round_trip():
    spec = synth.small_system(seed=14, order=3)
    # fast mode sums float atomics in scheduling order (like the reference); bitwise
    # repeatability is the deterministic mode's promise
    with make_box(spec, deterministic=1) as b:
        x0 = b.positions()
        assert np.array_equal(x0, spec.x.astype(np.float32))
        f1 = b.forces()
        f2 = b.forces()
        assert np.array_equal(f1, f2)
        assert np.array_equal(b.positions(), x0)


def test_rng_compat_mode_statistics():
    """cuRAND XORWOW mode (curand_init(seed, i, 0) + curand_normal): free particles with no
    forces diffuse with <dx^2> = 2 D dt per step under EM."""
    n = 4000
    rng = np.random.default_rng(0)
    L = 50.0
    spec = synth.SystemSpec("free", [L, L, L], [16, 16, 16], rng.uniform(10, 40, size=(n, 3)),
                            np.zeros(n, np.int32), ["A"], np.zeros((0, 2)), np.arange(n),
                            potentials=[], order=1, integrator="EM", delt=0.01)
    with make_box(spec, rng=1) as b:
        x0 = b.positions().astype(np.float64)
        b.step(10)
        x1 = b.positions().astype(np.float64)
    msd = ((x1 - x0) ** 2).mean()
    assert abs(msd - 10 * 2 * 0.01) < 0.05 * 10 * 2 * 0.01


def test_run_script_file_writes_ps_data(tmp_path):
    spec = synth.small_system(seed=15, order=3, charges=True)
    spec.log_freq = 10
    scr, _ = spec.write(str(tmp_path), steps=30)
    tild_b200.run_script_file(scr)
    rows = [l.split() for l in open(os.path.join(tmp_path, "ps_data.dat")) if l.strip()]
    # writeData(-1), steps 0, 10, 20, final writeData(30)
    assert [r[0] for r in rows] == ["-1", "0", "10", "20", "30"]
    assert all(len(r) == 2 + len(spec.potentials) for r in rows)   # step Ubond pot...
    assert os.path.exists(os.path.join(tmp_path, "final.input.data"))
    assert os.path.exists(os.path.join(tmp_path, "init.input.data"))


def test_nvt_log_matches_thermo():
    spec = synth.small_system(seed=16, order=3, charges=True)
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm)
    ref = oracle.pair_energies(sysm, dens)
    ub, _ = oracle.bond_energy(sysm)
    with make_box(spec) as b:
        b.run_nvt(3)
        log = b.log()
    assert log.shape[0] == 3   # -1, 0, final
    assert log[0, 0] == -1 and abs(log[0, 1] - ub) <= 1e-6 * abs(ub)
    for k, r in enumerate(ref):
        assert abs(log[0, 2 + k] - r) <= 1e-5 * abs(r)
    # step-0 row: pair energies from the step's start densities (x0), bonds after the update
    for k, r in enumerate(ref):
        assert abs(log[1, 2 + k] - r) <= 1e-5 * abs(r)


def test_ramp_updates_amplitude():
    spec = synth.small_system(seed=17, order=3)
    spec.potentials = [dict(kind="gaussian", I="A", J="B", A=2.0, sigma=0.7)]
    sysm = spec_to_system(spec)
    # ramp from 2 to 4 over 4 steps: after run_nvt(4) the amplitude is 4
    bb = tild_b200.Box(0, options={"write_files": 0})
    bb.command("Dim 3")
    bb.command("boxLengths %g %g %g" % tuple(spec.L))
    bb.command("grid %d %d %d" % tuple(spec.grid))
    bb.command("pmeorder %d" % spec.order)
    bb.command("randSeed %d" % spec.seed)
    bb.command("species A")
    bb.command("species B")
    bb.set_particles(spec.x, spec.types, spec.mol)
    bb.command("bond 1 harmonic 1.5 0.0")
    bb.set_bonds(spec.bonds)
    bb.command("potential gaussian A B 2.0 0.7 ramp 4.0")
    bb.command("integrator all GJF delt 0.005")
    bb.command("endBox")
    dens0, _, _ = oracle.densities(sysm)
    e2 = oracle.pair_energies(sysm, dens0)[0]
    t0 = bb.thermo()
    assert abs(t0["potentials"][0] - e2) <= 1e-5 * abs(e2), (t0["potentials"][0], e2)
    bb.run_nvt(4)
    log = bb.log()
    x = bb.positions()
    dens, _, _ = oracle.densities(sysm, x=x)
    e4 = oracle.pair_energies(sysm, dens)[0] * 2.0   # amplitude 4 = 2 x 2
    t = bb.thermo()
    assert abs(t["potentials"][0] - e4) <= 1e-5 * abs(e4)
    assert log.shape[0] == 3
    bb.close()


def test_full_size_c2_properties():
    """Coacervate at full size (2,097,152 particles, 192^3): momentum conservation of the
    grid forces and bonds (sum_p f_p ~ 0), finite forces, and a step that keeps every
    particle in the box."""
    spec = synth.config_c2()
    with make_box(spec) as b:
        f = b.forces().astype(np.float64)
        assert np.isfinite(f).all()
        frms = np.sqrt((f ** 2).sum(1).mean())
        assert np.abs(f.sum(0)).max() < 1e-4 * frms * np.sqrt(len(f))
        b.step(2)
        x = b.positions()
        assert (x >= 0).all() and (x <= spec.L).all()


@pytest.mark.parametrize("name", ["diblock_o3", "charged_o3", "erf", "odd_grid", "d2_charged"])
def test_pair_virial_and_pressure_match_oracle(name):
    """FP64 pair virial W_ab against the oracle (relative 1e-5 of max |W|), and the pressure
    tensor equal to (N kT delta + W_pair + W_bond)/V with kT = 1."""
    spec = SYSTEMS[name]()
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm)
    Wref = oracle.pair_virial(sysm, dens)
    with make_box(spec) as b:
        t = b.thermo()
    W = t["pair_virial"]
    assert np.abs(W - Wref).max() <= 1e-5 * np.abs(Wref).max(), (W, Wref)
    D = spec.dim
    V = float(np.prod(np.asarray(spec.L[:D], np.float64)))   # a 2-D box: its area
    P = (np.r_[np.full(D, spec.N), np.zeros(6 - D)] + W + t["virial"]) / V
    assert np.allclose(t["pressure"], P, rtol=1e-12, atol=0)


@pytest.mark.parametrize("charge", [False, True])
def test_structure_factor_matches_oracle(charge):
    spec = synth.small_system(seed=81, order=3, charges=True, grid=(15, 12, 18))
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm)
    group = "charges" if charge else "A"
    rho = dens[group][1] if charge else dens[group][0]
    kmax, nb = 8.0, 40
    kr, sr, nr = oracle.structure_factor(sysm, rho, nb, kmax)
    with make_box(spec) as b:
        k, sk, n = b.structure_factor(group, nb, kmax, charge=charge)
    assert np.array_equal(n, nr)
    assert np.allclose(k, kr, rtol=1e-12, atol=0)
    assert np.all(np.abs(sk - sr) <= 1e-5 * sr + 1e-7 * sr.max())


def test_angle_energy_and_resorting_with_angles():
    """Uangle against the FP64 oracle (1e-6 relative), and bit-identical trajectories in
    deterministic mode with re-sorting every step and never (angle slots renumbered)."""
    spec = SYSTEMS["angles"]()
    sysm = spec_to_system(spec)
    ua, _ = oracle.angle_energy(sysm)
    with make_box(spec) as b:
        t = b.thermo()
    assert abs(t["Uangle"] - ua) <= 1e-6 * abs(ua)
    outs = []
    for interval in (0, 1):
        with make_box(spec, deterministic=1, sort_interval=interval) as b:
            b.step(12)
            outs.append((b.positions(), b.forces()))
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])

