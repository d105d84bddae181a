"""CPU checks of the oracle itself: known answers, published test vectors, invariants.

The reference ships no tests or golden vectors; these pin the restatement to analytic
results, to the Philox paper's known-answer vectors, and (test_golden.py) to dumps of
the reference's own CUDA build when those fixtures exist."""
import numpy as np
import pytest

import oracle
from conftest import force_error, spec_to_system
from tild_b200 import synth


def test_philox_known_answers():
    # Random123 / Salmon et al. SC'11 known-answer vectors for philox4x32-10
    assert [int(v) for v in oracle.philox_raw([0, 0, 0, 0], [0, 0])] == \
        [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert [int(v) for v in oracle.philox_raw([0xffffffff] * 4, [0xffffffff] * 2)] == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert [int(v) for v in oracle.philox_raw([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                                              [0xa4093822, 0x299f31d0])] == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_philox_normals_moments():
    z = oracle.philox_normals(7, 3, np.arange(100000))
    assert np.all(np.abs(z.mean(0)) < 0.02)
    assert np.all(np.abs(z.std(0) - 1) < 0.02)


@pytest.mark.parametrize("order", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("prec", [32, 64])
def test_weights_partition_of_unity(order, prec):
    s = synth.small_system(seed=order, order=order)
    sysm = spec_to_system(s)
    inds, W = oracle.weights(sysm, prec=prec)
    _, _, gvol = oracle.grid_geometry(sysm)
    tol = 1e-5 if prec == 32 else 1e-12
    assert np.allclose(W.sum(1) * gvol, 1.0, atol=tol)
    assert inds.min() >= 0 and inds.max() < int(np.prod(sysm.Nx))


def test_order4_exact_is_quartic_bspline():
    """With quirk4=0 order 4 is the 5-point quartic B-spline (Deserno-Holm); with the
    reference's sx3 = sx2*sx2 (ps_grid_utils.cu:57) it is not."""
    s = synth.small_system(seed=4, order=4)
    sysm = spec_to_system(s, quirk4=0)
    sysm.L = np.full(3, 6.0, np.float32)            # isotropic: h = 0.5 in every direction
    rng = np.random.default_rng(0)
    L = float(sysm.L[0]); N = int(sysm.Nx[0]); h = L / N
    x = np.zeros((200, 3)); x[:, 0] = rng.uniform(0, L, 200); x[:, 1:] = h * 3  # y,z on nodes
    _, W = oracle.weights(sysm, x=x, prec=64)
    g = np.floor(x[:, 0] / h + 0.5)
    t = x[:, 0] / h - g          # in [-1/2, 1/2)

    def m5(u):                   # cardinal quartic B-spline centred at 0, support [-2.5, 2.5]
        u = np.abs(u)
        return np.where(u < 0.5, 115 / 192 - 5 / 8 * u ** 2 + u ** 4 / 4,
               np.where(u < 1.5, (55 + 20 * u - 120 * u ** 2 + 80 * u ** 3 - 16 * u ** 4) / 96,
               np.where(u < 2.5, (5 - 2 * u) ** 4 / 384, 0.0)))
    gvol = h ** 3
    Wx = W.reshape(200, 5, 5, 5)[:, :, 2, 2] * gvol / (m5(0.0) ** 2)
    ref = np.stack([m5(t + 2 - i) for i in range(5)], axis=1)
    assert np.allclose(Wx, ref, atol=1e-10)
    sysq = spec_to_system(s, quirk4=1)
    sysq.L = sysm.L
    _, Wq = oracle.weights(sysq, x=x, prec=64)
    assert not np.allclose(Wq, W)
    assert np.allclose(Wq.sum(1) * gvol, 1.0)


def test_fp32_mimic_vs_fp64_weights():
    s = synth.small_system(seed=3, order=3)
    sysm = spec_to_system(s)
    i32, w32 = oracle.weights(sysm, prec=32)
    i64, w64 = oracle.weights(sysm, prec=64)
    assert (i32 == i64).mean() > 0.999
    same = (i32 == i64).all(1)
    assert np.allclose(w32[same], w64[same], rtol=2e-6, atol=1e-7)


def test_net_force_vanishes():
    """Spectral ik-differentiation with identical assignment and interpolation conserves
    momentum: sum_p f_p = 0 up to round-off (the reference's logNetForce diagnostic,
    PS_Box.cu:320-335)."""
    s = synth.small_system(seed=5, charges=True)
    sysm = spec_to_system(s)
    f, _ = oracle.forces(sysm)
    assert np.abs(f.sum(0)).max() < 1e-10 * np.abs(f).max() * len(f)


def test_uniform_density_energy():
    """Particles on every node with order 0: rho uniform, U = A * rho^2 * V for a
    Gaussian with I != J (only k = 0 survives, u(0) = A)."""
    n = 6
    L = 6.0
    g = (np.arange(n) + 0.0) * (L / n)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1).astype(np.float32)
    types = np.r_[np.zeros(len(x) // 2), np.ones(len(x) - len(x) // 2)].astype(np.int32)
    x2 = np.concatenate([x, x])
    types2 = np.r_[np.zeros(len(x)), np.ones(len(x))].astype(np.int32)
    A = 1.7
    sysm = oracle.System(Dim=3, L=np.full(3, L, np.float32), Nx=np.full(3, n, np.int32), order=0,
                         x=x2, types=types2, mass=np.ones(2, np.float32), mobility=np.ones(2, np.float32),
                         species=["A", "B"],
                         potentials=[dict(kind="gaussian", I="A", J="B", A=A, sigma=0.5)])
    dens, _, _ = oracle.densities(sysm)
    E = oracle.pair_energies(sysm, dens)[0]
    rho = 1.0 / (L / n) ** 3
    assert abs(E - A * rho * rho * L ** 3) < 1e-9 * E
    f, _ = oracle.forces(sysm)
    assert np.abs(f).max() < 1e-9


@pytest.mark.parametrize("order", [1, 2, 3])
def test_isolated_particle_symmetric_self_force(order):
    L, n = 8.0, 16
    h = L / n
    # odd orders: cell centre is symmetric; even orders: grid node
    pos = (5 + 0.5) * h if order % 2 else 5 * h
    sysm = oracle.System(Dim=3, L=np.full(3, L, np.float32), Nx=np.full(3, n, np.int32), order=order,
                         x=np.full((1, 3), pos, np.float32), types=np.zeros(1, np.int32),
                         mass=np.ones(1, np.float32), mobility=np.ones(1, np.float32), species=["A"],
                         potentials=[dict(kind="gaussian", I="A", J="A", A=3.0, sigma=0.8)])
    f, _ = oracle.forces(sysm)
    assert np.abs(f).max() < 1e-10


def test_two_particle_force_converges_to_analytic():
    """Two particles in groups A and B with `potential gaussian A B`: the force on A
    approaches -d/dr of u(r) = A (2 pi s^2)^(-3/2) exp(-r^2 / 2 s^2) as the grid refines."""
    L, A, sig = 10.0, 2.0, 1.0
    xa = np.array([4.1, 5.2, 4.9]); xb = np.array([5.3, 4.6, 5.4])
    errs = []
    for n in (16, 32, 64):
        sysm = oracle.System(Dim=3, L=np.full(3, L, np.float32), Nx=np.full(3, n, np.int32), order=3,
                             x=np.stack([xa, xb]).astype(np.float32), types=np.array([0, 1], np.int32),
                             mass=np.ones(2, np.float32), mobility=np.ones(2, np.float32), species=["A", "B"],
                             potentials=[dict(kind="gaussian", I="A", J="B", A=A, sigma=sig)])
        f, _ = oracle.forces(sysm)
        r = (np.float32(xa) - np.float32(xb)).astype(np.float64)
        d = np.linalg.norm(r)
        u = A * (2 * np.pi * sig ** 2) ** -1.5 * np.exp(-d * d / (2 * sig ** 2))
        fa = u * r / sig ** 2      # -grad_a u
        errs.append(np.linalg.norm(f[0] - fa) / np.linalg.norm(fa))
        assert np.allclose(f[0], -f[1], atol=1e-12)
    # the spline smoothing of deposit + gather is an O(h^2) error: second-order convergence
    assert errs[0] > errs[1] > errs[2] and errs[2] < 0.03
    assert errs[1] / errs[2] > 3.0


@pytest.mark.parametrize("kind", ["erf2", "erfG"])
def test_erf_tables_small_k_limit(kind):
    pot = dict(kind=kind, A=1.3, Rp=1.0, sigma=0.5)
    k2 = np.array([0.0, 1e-8, 1e-6])
    u = oracle.uk(pot, k2)
    assert np.allclose(u[1:], u[0], rtol=1e-5)


def test_fp32_oracle_forces_match_fp64():
    s = synth.small_system(seed=9, charges=True)
    sysm = spec_to_system(s)
    f64, _ = oracle.forces(sysm, prec=64)
    f32, _ = oracle.forces(sysm, prec=32)
    assert force_error(f32, f64) < 1e-5


def test_gjf_trajectory_fp32_vs_fp64():
    s = synth.small_system(seed=2)
    sysm = spec_to_system(s)
    t64 = oracle.Trajectory(sysm, 64)
    t32 = oracle.Trajectory(sysm, 32)
    for step in range(20):
        nz = oracle.philox_normals(17, step, np.arange(sysm.N))
        t64.step(nz)
        t32.step(nz)
    d = np.abs(t64.positions() - t32.positions())
    d = np.minimum(d, sysm.L - d)
    assert d.max() < 1e-4


def _energy_scaled(sysm, dens, scale):
    """Total pair energy, FP64, after an affine stretch of the box by `scale` per axis.
    The grid follows the box, so each field's weight sums rho * gvol stay fixed."""
    glist = oracle.groups(sysm)
    Nx = sysm.Nx.astype(np.int64)
    shape = tuple(int(v) for v in Nx[::-1])
    M = int(np.prod(Nx))
    L0 = sysm.L.astype(np.float32).astype(np.float64)
    L = L0 * np.asarray(scale, np.float64)
    gvol0, gvol = float(np.prod(L0 / Nx)), float(np.prod(L / Nx))
    ks = []
    for d in range(3):
        n = np.arange(Nx[d])
        k = 2.0 * np.pi * np.where(n < Nx[d] / 2.0, n, n - Nx[d]) / L[d]
        s = [1, 1, 1]
        s[2 - d] = int(Nx[d])
        ks.append(k.reshape(s))
    k2 = ks[0] ** 2 + ks[1] ** 2 + ks[2] ** 2
    U = 0.0
    for pot in sysm.potentials:
        if pot["kind"] == "charges":
            rI = rJ = dens["charges"][1]
            fac = 0.5
        else:
            rI = dens[glist[oracle.find_group(glist, pot["I"])][0]][0]
            rJ = dens[glist[oracle.find_group(glist, pot["J"])][0]][0]
            fac = 1.0
        fI = np.fft.fftn(rI.astype(np.float64).reshape(shape) * gvol0 / gvol) / M
        fJ = np.fft.fftn(rJ.astype(np.float64).reshape(shape) * gvol0 / gvol) / M
        U += fac * gvol * M * float(np.sum(np.broadcast_to(oracle.uk(pot, k2), shape) * (np.conj(fI) * fJ).real))
    return U


@pytest.mark.parametrize("kind", ["gaussian", "charges", "erf"])
def test_pair_virial_is_the_strain_derivative_of_the_energy(kind):
    """W_aa = -dU/d(strain_aa): the FP64 pair virial against central differences of the
    pair energy under stretching the box along each axis (relative 1e-7)."""
    if kind == "erf":
        spec = synth.small_system(seed=71, order=3, pots=[
            dict(kind="erf2", I="A", J="B", A=0.05, Rp=1.0, sigma=0.5),
            dict(kind="erfG", I="B", J="B", A=0.3, Rp=0.8, sigma=0.5)])
    else:
        spec = synth.small_system(seed=72, order=3, charges=(kind == "charges"))
    sysm = spec_to_system(spec)
    dens, _, _ = oracle.densities(sysm)
    W = oracle.pair_virial(sysm, dens)
    assert abs(_energy_scaled(sysm, dens, [1, 1, 1]) - sum(oracle.pair_energies(sysm, dens))) <= 1e-9 * abs(W[:3]).max()
    h = 1e-5
    for a in range(3):
        sp, sm = np.ones(3), np.ones(3)
        sp[a], sm[a] = 1 + h, 1 - h
        fd = -(_energy_scaled(sysm, dens, sp) - _energy_scaled(sysm, dens, sm)) / (2 * h)
        assert abs(W[a] - fd) <= 1e-7 * abs(W[:3]).max(), (kind, a, W[a], fd)


ANGLES = [dict(style="harmonic", k=3.0, theta=120.0), dict(style="wlc", k=2.0)]


def test_angle_forces_are_the_energy_gradient():
    """Oracle angle forces (ps_deviceAngles.cu formulas) = -grad of the angle energy, FP64
    central differences on random chain geometries, both styles."""
    spec = synth.small_system(seed=91, order=3, angle_params=ANGLES)
    sysm = spec_to_system(spec)
    fi, fk, _, _ = oracle.angle_terms(sysm)
    a = np.asarray(sysm.angles)
    f = np.zeros((sysm.N, 3))
    np.add.at(f, a[:, 0], fi)
    np.add.at(f, a[:, 1], -(fi + fk))
    np.add.at(f, a[:, 2], fk)
    x0 = sysm.x.astype(np.float64)
    h = 1e-6
    for p in (0, 1, 3, 7, 9, 40):
        for d in range(3):
            xp, xm = x0.copy(), x0.copy()
            xp[p, d] += h
            xm[p, d] -= h
            g = (oracle.angle_energy(sysm, xp)[0] - oracle.angle_energy(sysm, xm)[0]) / (2 * h)
            assert abs(-g - f[p, d]) <= 1e-6 * (1 + abs(f[p, d])), (p, d, -g, f[p, d])


def test_angle_script_and_data_file_round_trip(tmp_path):
    """angle words, the Angles section and MAXANGLES are read like readInput/readDataConfig."""
    import tild_b200
    spec = synth.small_system(seed=92, order=3, angle_params=ANGLES)
    scr, data = spec.write(str(tmp_path), steps=0)
    b = tild_b200.Box(base_dir=str(tmp_path), options={"write_files": 0})
    for line in open(scr).read().split("endBox")[0].splitlines()[1:]:   # the words after "box ps"
        if line.strip():
            b.command(line)
    d = b.describe()
    assert d["nAngles"] == len(spec.angles)
    b.close()
