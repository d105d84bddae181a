"""CPU oracle for the TILD particle-mesh step (test infrastructure only).

This module is the checker for the CUDA product under ``matilda.ft_b200/`` and the
CPU baseline timed by ``bench.py``.  The product never imports it.  It restates the
reference MATILDA.FT ``PS_Box`` step (paths relative to the MATILDA.FT source tree):

* stencil indices/weights   ps_grid_utils.cu:17-204        (C, tild_oracle.c)
* density deposit           device_utils.cu:282-352        (C)
* spectral forces           ps_potential.cu:41-125, Box.cu:107-127 (numpy FFT)
* potential tables          ps_potentialGaussian.cu:28-46, ps_potentialErf2.cu:101-124,
                            ps_potentialErfG.cu:167-190, ps_potentialCharges.cu:231-258
* k vectors                 Box.cu:133-178
* grid -> particle forces   device_utils.cu:358-461        (C)
* bonds, bond energy        ps_deviceBonds.cu:7-171        (C)
* GJF / EM                  ps_integratorGJF.cu:43-163, ps_integratorEM.cu:39-82 (C)
* pair energies             ps_potential.cu:133-178, ps_potentialCharges.cu:274-322
* step order                PS_Box.cu:73-278

FFT: the reference calls cuFFT C2C FP32 (CUDA toolkit; no version pinned by the
reference, 12.9.86 in this image).  cuFFT's internals are unpublished; the oracle uses
the DFT definition through numpy.fft (pocketfft, FP64): forward e^{-2 pi i k.r},
normalised by 1/M after the forward transform, inverse unnormalised, real part kept.

Parity pinning: the reference ships no tests or golden vectors.  The oracle is pinned
(a) by the analytic known answers in tests/test_oracle.py and (b) against dumps of the
reference's own CUDA build when tests/golden/ref_*.npz exist (made by
oracle/ref_harness on a GPU).  Without (b) parity is unpinned.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def _lib(prec: int):
    if prec not in _LIBS:
        path = os.path.join(_HERE, "lib", "liborc%d.so" % prec)
        if not os.path.exists(path):
            import subprocess
            subprocess.run(["make", "-s", "-C", _HERE], check=True)
        _LIBS[prec] = ctypes.CDLL(path)
    return _LIBS[prec]


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


PI2_F32 = np.float32(6.2831853071)  # constants.h:9
PI4 = 12.56637061435917295384      # constants.h:10


@dataclass
class System:
    """Plain description of one PS box (what readInput + readDataConfig produce)."""
    Dim: int
    L: np.ndarray            # float32[Dim]
    Nx: np.ndarray           # int32[Dim]
    order: int               # pmeorder
    x: np.ndarray            # float32[N, Dim]
    types: np.ndarray        # int32[N], 0-based species index
    mass: np.ndarray         # float32[ntypes]
    mobility: np.ndarray     # float32[ntypes]
    species: list            # labels
    charges: np.ndarray | None = None   # float32[N] when doCharges
    nb: np.ndarray | None = None        # int32[N]
    partner: np.ndarray | None = None   # int32[N, maxb]
    btype: np.ndarray | None = None     # int32[N, maxb]
    bond_k: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    bond_req: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    bond_style: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    potentials: list = field(default_factory=list)  # dicts: kind,I,J,A,sigma,Rp,lB
    user_groups: list = field(default_factory=list)  # (name, [species labels])
    quirk4: int = 1
    delt: float = 0.005
    integrator: str = "GJF"
    integ_group: str = "all"
    angles: np.ndarray | None = None        # int[na, 3]: i, middle j, k (0-based)
    angle_types: np.ndarray | None = None   # int[na]
    angle_k: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    angle_theq: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))   # radians
    angle_style: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))    # 0 wlc, 1 harmonic

    @property
    def N(self):
        return self.x.shape[0]

    @property
    def maxb(self):
        return 0 if self.partner is None else self.partner.shape[1]


def groups(sysm: System):
    """Group list in the reference's order: user groups (pushed while parsing,
    PS_Box_initialization.cu:194-197), then all, one per species, charges
    (createDefaultGroups, PS_Box_initialization.cu:573-587)."""
    out = []
    for name, labels in sysm.user_groups:
        tids = [sysm.species.index(lb) for lb in labels]
        out.append((name, np.nonzero(np.isin(sysm.types, tids))[0].astype(np.int32), False))
    out.append(("all", np.arange(sysm.N, dtype=np.int32), False))
    for t, lb in enumerate(sysm.species):
        out.append((lb, np.nonzero(sysm.types == t)[0].astype(np.int32), False))
    if sysm.charges is not None:
        out.append(("charges", np.nonzero(sysm.charges != 0)[0].astype(np.int32), True))
    return out


def find_group(glist, name):
    for i, g in enumerate(glist):
        if g[0] == name:
            return i
    raise KeyError(name)


def grid_geometry(sysm: System):
    """dx in double from float L (PS_Box_initialization.cu:377-380), dxf = (float)dx
    (:727-731), gvol double (:379) and its float32 conversion used by the gathers."""
    L = sysm.L.astype(np.float32)
    dx = L.astype(np.float64) / sysm.Nx.astype(np.float64)
    dxf = dx.astype(np.float32)
    gvol = float(np.prod(dx))
    return dx, dxf, gvol


def weights(sysm: System, x=None, prec=64):
    """Per-particle stencil indices and weights (d_calcGridWeights)."""
    x = sysm.x if x is None else x
    real = np.float32 if prec == 32 else np.float64
    lib = _lib(prec)
    dx, dxf, _ = grid_geometry(sysm)
    G = (sysm.order + 1) ** sysm.Dim
    n = x.shape[0]
    xs = np.ascontiguousarray(x, dtype=real)
    d = (dxf if prec == 32 else dx).astype(real)
    nx = np.ascontiguousarray(sysm.Nx, dtype=np.int32)
    inds = np.zeros(n * G, np.int32)
    W = np.zeros(n * G, real)
    getattr(lib, "orc%d_grid_weights" % prec)(
        ctypes.c_int(n), _p(xs), ctypes.c_int(sysm.Dim), _p(nx), _p(d),
        ctypes.c_int(sysm.order), ctypes.c_int(sysm.quirk4), _p(inds), _p(W))
    return inds.reshape(n, G), W.reshape(n, G)


def kvectors(sysm: System, prec=64):
    """k_d = 2 pi n/L_d for n < N_d/2 else 2 pi (n - N_d)/L_d (Box.cu:157-178),
    as an array per dimension, broadcast to the grid shape (z, y, x)."""
    ks = []
    for d in range(sysm.Dim):
        N = int(sysm.Nx[d])
        n = np.arange(N)
        nn = np.where(n.astype(np.float64) < N / 2.0, n, n - N)
        if prec == 32:
            k = (PI2_F32 * nn.astype(np.float32)) / np.float32(sysm.L[d])
        else:
            k = 2.0 * np.pi * nn / float(sysm.L[d])
        ks.append(k)
    shape = [int(v) for v in sysm.Nx[::-1]]
    out = []
    for d in range(sysm.Dim):
        s = [1] * sysm.Dim
        s[sysm.Dim - 1 - d] = shape[sysm.Dim - 1 - d]
        out.append(np.broadcast_to(ks[d].reshape(s), shape))
    return out


def uk(pot, k2):
    """û(k) of each pair potential kind (FP64)."""
    kind = pot["kind"]
    if kind == "gaussian":   # ps_potentialGaussian.cu:38-46
        return pot["A"] * np.exp(-k2 * pot["sigma"] ** 2 / 2.0)
    if kind in ("erf2", "erfG"):  # ps_potentialErf2.cu:111-124, ps_potentialErfG.cu:177-190
        Rp = pot["Rp"]
        k = np.sqrt(k2)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = PI4 * (np.sin(Rp * k) - Rp * k * np.cos(Rp * k)) / (k2 * k)
        t0 = PI4 * Rp ** 3 / 3.0
        t = np.where(k2 == 0.0, t0, t)
        g = np.exp(-k2 * pot["sigma"] ** 2 * 0.5)
        if kind == "erf2":
            return np.where(k2 == 0.0, pot["A"] * t0 * t0, pot["A"] * g * t * t)
        return np.where(k2 == 0.0, pot["A"] * t0, pot["A"] * g * t)
    if kind == "charges":    # ps_potentialCharges.cu:241-258
        with np.errstate(divide="ignore", invalid="ignore"):
            u = PI4 * pot["lB"] / k2 * np.exp(-k2 * pot["sigma"] ** 2)
        return np.where(k2 > 0.0, u, 0.0)
    raise ValueError(kind)


def duk_over_k(pot, k2):
    """(d û/dk)/k of each kind (FP64), 0 at k = 0: the strain derivative of û."""
    kind = pot["kind"]
    pos = k2 > 0.0
    with np.errstate(divide="ignore", invalid="ignore"):
        if kind == "gaussian":
            return -pot["sigma"] ** 2 * uk(pot, k2)
        if kind == "charges":
            return np.where(pos, uk(pot, k2) * (-2.0 * pot["sigma"] ** 2 - 2.0 / k2), 0.0)
        if kind in ("erf2", "erfG"):
            R, s2 = pot["Rp"], pot["sigma"] ** 2
            k = np.sqrt(k2)
            f = np.sin(R * k) - R * k * np.cos(R * k)
            t = PI4 * f / (k2 * k)
            dt_k = PI4 * (R * R * np.sin(R * k) / (k2 * k) - 3.0 * f / (k2 * k2 * k))
            g = np.exp(-0.5 * k2 * s2)
            if kind == "erf2":
                v = pot["A"] * g * t * (-s2 * t + 2.0 * dt_k)
            else:
                v = pot["A"] * g * (-s2 * t + dt_k)
            return np.where(pos, v, 0.0)
    raise ValueError(kind)


def pair_virial(sysm: System, dens):
    """Pair virial W_ab = -dU_pair/d(strain_ab) for an affine strain of the box and the
    positions (the grid follows the box, so the deposited weights do not change):
    U = C/V sum_k û(|k|) Re(rho_I* rho_J) gives W_ab = U delta_ab + C/V sum_k (û'(k)/k)
    k_a k_b Re(rho_I* rho_J).  Components xx, yy, zz, xy, xz, yz (FP64; those with z are 0
    in a 2-D box)."""
    glist = groups(sysm)
    shape = _grid_shape(sysm)
    M = int(np.prod(sysm.Nx))
    ks = kvectors(sysm, 64)
    k2 = sum(k * k for k in ks)
    _, _, gvol = grid_geometry(sysm)
    W = np.zeros(6)
    utot = 0.0
    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
    for pot in kspace_potentials(sysm):
        if pot["kind"] == "charges":
            rI = rJ = dens["charges"][1]
            fac = 0.5
        else:
            rI = dens[glist[find_group(glist, pot["I"])][0]][0]
            rJ = dens[glist[find_group(glist, pot["J"])][0]][0]
            fac = 1.0
        fI = np.fft.fftn(rI.astype(np.float64).reshape(shape)) / M
        fJ = np.fft.fftn(rJ.astype(np.float64).reshape(shape)) / M
        re = (np.conj(fI) * fJ).real
        c = fac * gvol * M
        utot += c * float(np.sum(uk(pot, k2) * re))
        d = duk_over_k(pot, k2) * re
        for i, (a, b) in enumerate(pairs):
            if a < sysm.Dim and b < sysm.Dim:   # a 2-D box has only xx, yy, xy
                W[i] += c * float(np.sum(d * ks[a] * ks[b]))
    W[:sysm.Dim] += utot
    return W


def structure_factor(sysm: System, rho, nbins: int, kmax: float):
    """S(k) = |FFT(rho)/M|^2 over every k-vector of the grid (ps_compute_sk.cu:18-50),
    averaged in nbins shells of |k| (width kmax/nbins), k_d = (2 pi/L_d) n_d with the
    signed index of Box.cu:157-178.  Returns (mean |k|, mean S, count) per shell, FP64."""
    shape = _grid_shape(sysm)
    M = int(np.prod(sysm.Nx))
    f = np.fft.fftn(np.asarray(rho, np.float64).reshape(shape)) / M
    S = (f.real ** 2 + f.imag ** 2).reshape(-1)
    ks = []
    for d in range(3):
        N = int(sysm.Nx[d])
        n = np.arange(N)
        k = (2.0 * np.pi / float(np.float32(sysm.L[d]))) * np.where(n < N - n, n, n - N)
        s = [1, 1, 1]
        s[2 - d] = N
        ks.append(k.reshape(s))
    kk = np.sqrt(np.broadcast_to(ks[0] ** 2 + ks[1] ** 2 + ks[2] ** 2, shape)).reshape(-1)
    b = np.floor(kk * (nbins / kmax)).astype(np.int64)
    ok = b < nbins
    cnt = np.bincount(b[ok], minlength=nbins).astype(np.float64)
    ssum = np.bincount(b[ok], weights=S[ok], minlength=nbins)
    ksum = np.bincount(b[ok], weights=kk[ok], minlength=nbins)
    with np.errstate(invalid="ignore", divide="ignore"):
        return (np.where(cnt > 0, ksum / cnt, (np.arange(nbins) + 0.5) * kmax / nbins),
                np.where(cnt > 0, ssum / cnt, 0.0), cnt)


def _grid_shape(sysm):
    return tuple(int(v) for v in sysm.Nx[::-1])


def densities(sysm: System, x=None, prec=64):
    """Every group's rho (and rhoq for 'charges'): PS_Box.cu:108-114."""
    x = sysm.x if x is None else x
    real = np.float32 if prec == 32 else np.float64
    lib = _lib(prec)
    inds, W = weights(sysm, x, prec)
    G = inds.shape[1]
    M = int(np.prod(sysm.Nx))
    q = None if sysm.charges is None else np.ascontiguousarray(sysm.charges, dtype=real)
    out = {}
    for name, sites, is_q in groups(sysm):
        rho = np.zeros(M, real)
        rhoq = np.zeros(M, real) if is_q else None
        getattr(lib, "orc%d_deposit" % prec)(
            ctypes.c_int(len(sites)), _p(sites), ctypes.c_int(G), _p(inds), _p(W),
            _p(q) if is_q else None, _p(rho), _p(rhoq), ctypes.c_int(1))
        out[name] = (rho, rhoq)
    return out, inds, W


def spectral_grid_forces(sysm: System, dens, prec=64):
    """gridForce[group] (Dim, M) from every potential's CalcForces
    (ps_potential.cu:41-125; ps_potentialCharges.cu:328-368)."""
    glist = groups(sysm)
    shape = _grid_shape(sysm)
    M = int(np.prod(sysm.Nx))
    ks = kvectors(sysm, 64)
    k2 = sum(k * k for k in ks)
    gf = {}
    for pot in kspace_potentials(sysm):
        u = uk(pot, k2)
        if pot["kind"] == "charges":
            I = J = find_group(glist, "charges")
            rhoJ = dens["charges"][1]
            sides = [(I, rhoJ, 1.0)]
        else:
            I = find_group(glist, pot["I"])
            J = find_group(glist, pot["J"])
            sides = [(I, dens[glist[J][0]][0], 2.0 if I == J else 1.0)]
            if I != J:
                sides.append((J, dens[glist[I][0]][0], 1.0))
        for tgt, rho, mult in sides:
            rk = np.fft.fftn(rho.astype(np.float64).reshape(shape)) / M
            acc = gf.setdefault(tgt, np.zeros((sysm.Dim, M)))
            for d in range(sysm.Dim):
                fk = -1j * ks[d] * u
                g = np.fft.ifftn(fk * rk).real * M
                acc[d] += mult * g.reshape(M)
    return gf


def angle_terms(sysm: System, x=None):
    """Per angle (FP64): forces fi on i and fk on k (the middle particle takes
    -(fi + fk)), energy and virial r_ij,a f_i,b + r_kj,a f_k,b (xx, yy, zz, xy, xz, yz), as
    ps_deviceAngles.cu:26-120 and 151-294 compute them: minimum image with L/2, angles with
    a bond shorter than 1e-2 skipped, wlc U = k (1 + cos), harmonic U = k (theta - theta_eq)^2
    (skipped for |cos| > 1, 1/sin taken as 0 below 1e-4)."""
    x = np.asarray(sysm.x if x is None else x, np.float64)
    a = np.asarray(sysm.angles, np.int64)
    t = np.asarray(sysm.angle_types, np.int64)
    L = np.asarray(sysm.L, np.float32).astype(np.float64)
    Lh = (0.5 * np.asarray(sysm.L, np.float32)).astype(np.float64)

    def mi(d):
        return np.where(d > Lh, d - L, np.where(d < -Lh, d + L, d))

    rij = mi(x[a[:, 0]] - x[a[:, 1]])
    rkj = mi(x[a[:, 2]] - x[a[:, 1]])
    m2i, m2k = (rij * rij).sum(1), (rkj * rkj).sum(1)
    ok = (m2i >= 1e-4) & (m2k >= 1e-4)
    mi_, mk = np.sqrt(m2i), np.sqrt(m2k)
    with np.errstate(divide="ignore", invalid="ignore"):
        cos = (rij * rkj).sum(1) / mi_ / mk
        k = np.asarray(sysm.angle_k, np.float64)[t]
        wlc = np.asarray(sysm.angle_style)[t] == 0
        dri = rkj / (mi_ * mk)[:, None] - (cos / m2i)[:, None] * rij
        drk = rij / (mi_ * mk)[:, None] - (cos / m2k)[:, None] * rkj
        theta = np.arccos(np.clip(cos, -1.0, 1.0))
        den = np.sqrt(np.maximum(1.0 - cos * cos, 0.0))
        isin = np.where(den > 1e-4, 1.0 / den, 0.0)
        dth = theta - np.asarray(sysm.angle_theq, np.float64)[t]
        coef = np.where(wlc, -k, 2.0 * k * dth * isin)
        e = np.where(wlc, k * (1.0 + cos), k * dth * dth)
        ok &= wlc | ((cos >= -1.0) & (cos <= 1.0))
    fi = np.where(ok[:, None], coef[:, None] * dri, 0.0)
    fk = np.where(ok[:, None], coef[:, None] * drk, 0.0)
    e = np.where(ok, e, 0.0)
    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
    D = rij.shape[1]   # components with z are 0 in a 2-D box
    vir = np.stack([fi[:, p] * rij[:, q] + fk[:, p] * rkj[:, q] if p < D and q < D else np.zeros(len(e))
                    for p, q in pairs], 1)
    return fi, fk, e, vir


def angle_energy(sysm: System, x=None):
    """Uangle and the angle virial sum (FP64)."""
    if sysm.angles is None or len(sysm.angles) == 0:
        return 0.0, np.zeros(6)
    _, _, e, vir = angle_terms(sysm, x)
    return float(e.sum()), vir.sum(0)


AXES = {"x": 0, "X": 0, "y": 1, "Y": 1, "z": 2, "Z": 2}


def wall_terms(sysm: System, pot, x=None, real=np.float64):
    """Harmonic wall (ps_potentialWall.cu:92-131) on group I: per site, the force
    k (pos - x_axis) along the axis and the energy k disp^2 / 2 where sign (pos - x_axis) > 0.
    Returns (sites, axis, force per site, energy per site)."""
    x = sysm.x if x is None else x
    glist = groups(sysm)
    sites = glist[find_group(glist, pot["I"])][1]
    a = AXES[pot["axis"]]
    xs = np.asarray(x, real).reshape(sysm.N, sysm.Dim)[sites, a]
    disp = real(pot["pos"]) - xs
    on = real(pot["sign"]) * disp > 0
    k = real(pot["k"])
    return sites, a, np.where(on, k * disp, 0), np.where(on, real(0.5) * k * disp * disp, 0)


def kspace_potentials(sysm: System):
    """The potentials that act through the grid (every kind but the per-particle wall)."""
    return [p for p in sysm.potentials if p["kind"] != "wall"]


def forces(sysm: System, x=None, prec=64, include_bonds=True, include_grid=True):
    """Total force on every particle: bonds, then each force group's gather in the
    reference's group order (PS_Box.cu:240-270).  Returns f[N, Dim] (float64 for
    prec=64) and a dict of intermediates."""
    x = sysm.x if x is None else x
    real = np.float32 if prec == 32 else np.float64
    lib = _lib(prec)
    N, Dim = sysm.N, sysm.Dim
    f = np.zeros(N * Dim, real)
    xs = np.ascontiguousarray(x, dtype=real).reshape(-1)
    Lr = np.ascontiguousarray(sysm.L, dtype=real)
    if include_bonds and sysm.partner is not None:
        getattr(lib, "orc%d_bonds" % prec)(
            ctypes.c_int(N), ctypes.c_int(Dim), _p(xs), _p(sysm.nb), _p(sysm.partner),
            _p(sysm.btype), ctypes.c_int(sysm.maxb), _p(sysm.bond_k.astype(real)),
            _p(sysm.bond_req.astype(real)), _p(sysm.bond_style.astype(np.int32)), _p(Lr), _p(f))
    if include_bonds and sysm.angles is not None and len(sysm.angles):   # after the bonds (PS_Box.cu:245-254)
        fi, fk, _, _ = angle_terms(sysm, x)
        fa = np.zeros((N, Dim))
        a = np.asarray(sysm.angles, np.int64)
        np.add.at(fa, a[:, 0], fi)
        np.add.at(fa, a[:, 1], -(fi + fk))
        np.add.at(fa, a[:, 2], fk)
        f += fa.reshape(-1).astype(real)
    for pot in sysm.potentials:   # walls add to the forces before the gathers (PS_Box.cu:262-264)
        if include_grid and pot["kind"] == "wall":
            sites, ax, fw, _ = wall_terms(sysm, pot, x, real)
            fv = f.reshape(N, Dim)
            fv[sites, ax] += fw
    inter = {}
    if include_grid:
        dens, inds, W = densities(sysm, x, prec)
        gf = spectral_grid_forces(sysm, dens, prec)
        _, _, gvol = grid_geometry(sysm)
        glist = groups(sysm)
        G = inds.shape[1]
        q = None if sysm.charges is None else np.ascontiguousarray(sysm.charges, dtype=real)
        # force flags: groups named by a non-charge potential, plus 'charges'
        flagged = set()
        for pot in kspace_potentials(sysm):
            if pot["kind"] != "charges":
                flagged.add(find_group(glist, pot["I"]))
                flagged.add(find_group(glist, pot["J"]))
        for gi, (name, sites, is_q) in enumerate(glist):
            if gi not in flagged and not is_q:
                continue
            grid = gf.get(gi, np.zeros((Dim, int(np.prod(sysm.Nx)))))
            gridF = np.ascontiguousarray(grid.T.astype(real))  # [M, Dim] interleaved
            getattr(lib, "orc%d_gather" % prec)(
                ctypes.c_int(len(sites)), _p(sites), ctypes.c_int(G), _p(inds), _p(W),
                (ctypes.c_float if prec == 32 else ctypes.c_double)(
                    np.float32(gvol) if prec == 32 else gvol),
                _p(gridF), _p(q) if is_q else None, ctypes.c_int(Dim), _p(f))
        inter = dict(dens=dens, gridforce=gf, inds=inds, W=W)
    return f.reshape(N, Dim), inter


def pair_energies(sysm: System, dens, x=None):
    """Per-potential energy: gvol * sum rho_I (u*rho_J) (ps_potential.cu:133-178, no
    1/2 for I==J); charges 0.5*gvol*sum rhoq (u*rhoq) (ps_potentialCharges.cu:274-322)."""
    glist = groups(sysm)
    shape = _grid_shape(sysm)
    M = int(np.prod(sysm.Nx))
    ks = kvectors(sysm, 64)
    k2 = sum(k * k for k in ks)
    _, _, gvol = grid_geometry(sysm)
    out = []
    for pot in sysm.potentials:
        if pot["kind"] == "wall":   # Wall::CalcEnergy (ps_potentialWall.cu:58-70) at the positions
            out.append(float(np.sum(wall_terms(sysm, pot, x)[3])))
            continue
        u = uk(pot, k2)
        if pot["kind"] == "charges":
            rI = rJ = dens["charges"][1]
            fac = 0.5
        else:
            rI = dens[glist[find_group(glist, pot["I"])][0]][0]
            rJ = dens[glist[find_group(glist, pot["J"])][0]][0]
            fac = 1.0
        rk = np.fft.fftn(rJ.astype(np.float64).reshape(shape)) / M
        conv = np.fft.ifftn(u * rk).real * M
        out.append(fac * gvol * float(np.sum(rI.astype(np.float64).reshape(shape) * conv)))
    return out


def bond_energy(sysm: System, x=None, prec=64):
    """Ubond = 0.5 * sum of per-particle energies (PS_Box.cu:284-292) and the summed
    virial components."""
    x = sysm.x if x is None else x
    if sysm.partner is None:
        return 0.0, np.zeros(6)
    real = np.float32 if prec == 32 else np.float64
    lib = _lib(prec)
    N, Dim = sysm.N, sysm.Dim
    npc = 3 if Dim == 2 else 6
    e = np.zeros(N, real)
    vir = np.zeros(N * npc, real)
    xs = np.ascontiguousarray(x, dtype=real).reshape(-1)
    getattr(lib, "orc%d_bond_energy" % prec)(
        ctypes.c_int(N), ctypes.c_int(Dim), _p(xs), _p(sysm.nb), _p(sysm.partner),
        _p(sysm.btype), ctypes.c_int(sysm.maxb), _p(sysm.bond_k.astype(real)),
        _p(sysm.bond_req.astype(real)), _p(sysm.bond_style.astype(np.int32)),
        _p(np.ascontiguousarray(sysm.L, dtype=real)), _p(e), _p(vir))
    return 0.5 * float(np.sum(e.astype(np.float64))), vir.reshape(N, npc).sum(0)


def philox_normals(seed: int, step: int, ids):
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    out = np.zeros(3 * len(ids), np.float32)
    _lib(64).orc_philox_normals(ctypes.c_uint64(seed), ctypes.c_uint32(step),
                                ctypes.c_int(len(ids)), _p(ids), _p(out))
    return out.reshape(-1, 3)


def philox_raw(ctr, key):
    c = np.ascontiguousarray(ctr, dtype=np.uint32).copy()
    k = np.ascontiguousarray(key, dtype=np.uint32)
    _lib(64).orc_philox4x32_10(_p(c), _p(k))
    return c


class CpuStep:
    """The reference's step run on the host cores, FP32 like the reference: stencil
    tables for every particle, a deposit into EVERY group (PS_Box.cu:108-114), one FP32
    C2C forward FFT per potential side and three inverse C2C FFTs per force direction
    (ps_potential.cu:41-125), gathers, bonds and GJF.  FFTs use scipy.fft (pocketfft)
    on `threads` workers; the C loops use OpenMP with `threads` threads.  This is the
    timed CPU baseline, not a checker."""

    def __init__(self, sysm: System, threads: int, seed: int = 1):
        import scipy.fft
        self.fft = scipy.fft
        self.s = sysm
        self.threads = threads
        self.lib = _lib(32)
        self.x = np.ascontiguousarray(sysm.x, np.float32).reshape(-1).copy()
        self.xo = self.x.copy()
        self.old_noise = np.zeros_like(self.x)
        self.glist = groups(sysm)
        self.sites = self.glist[find_group(self.glist, sysm.integ_group)][1]
        self.shape = _grid_shape(sysm)
        self.M = int(np.prod(sysm.Nx))
        ks = kvectors(sysm, 32)
        k2 = sum(k.astype(np.float64) ** 2 for k in ks)
        if any(p["kind"] == "wall" for p in sysm.potentials):
            raise NotImplementedError("CpuStep times grid potentials only; Trajectory covers walls")
        self.fk = []
        for pot in sysm.potentials:   # host tables built once, FP32 complex (fk = -i k u)
            u = uk(pot, k2).astype(np.float32)
            self.fk.append([(-1j * ks[d] * u).astype(np.complex64) for d in range(sysm.Dim)])
        self.seed = seed
        self.step_i = 0
        self.q = None if sysm.charges is None else np.ascontiguousarray(sysm.charges, np.float32)
        _, _, self.gvol = grid_geometry(sysm)

    def _fwd(self, rho):
        a = rho.reshape(self.shape).astype(np.complex64)
        return self.fft.fftn(a, workers=self.threads) * np.float32(1.0 / self.M)

    def _inv(self, a):
        return (self.fft.ifftn(a, workers=self.threads, norm="forward")).real.astype(np.float32)

    def step(self):
        s, lib, th = self.s, self.lib, self.threads
        N, Dim, M = s.N, s.Dim, self.M
        _, dxf, _ = grid_geometry(s)
        G = (s.order + 1) ** Dim
        inds = np.empty(N * G, np.int32)
        W = np.empty(N * G, np.float32)
        lib.orc32_grid_weights(ctypes.c_int(N), _p(self.x), ctypes.c_int(Dim),
                               _p(np.ascontiguousarray(s.Nx, np.int32)), _p(dxf.astype(np.float32)),
                               ctypes.c_int(s.order), ctypes.c_int(s.quirk4), _p(inds), _p(W))
        dens = {}
        for name, sites, is_q in self.glist:
            rho = np.zeros(M, np.float32)
            rhoq = np.zeros(M, np.float32) if is_q else None
            lib.orc32_deposit(ctypes.c_int(len(sites)), _p(sites), ctypes.c_int(G), _p(inds), _p(W),
                              _p(self.q) if is_q else None, _p(rho), _p(rhoq), ctypes.c_int(th))
            dens[name] = (rho, rhoq)
        f = np.zeros(N * Dim, np.float32)
        Lr = np.ascontiguousarray(s.L, np.float32)
        if s.partner is not None:
            lib.orc32_bonds(ctypes.c_int(N), ctypes.c_int(Dim), _p(self.x), _p(s.nb), _p(s.partner),
                            _p(s.btype), ctypes.c_int(s.maxb), _p(s.bond_k.astype(np.float32)),
                            _p(s.bond_req.astype(np.float32)), _p(s.bond_style.astype(np.int32)), _p(Lr), _p(f))
        gf = {}
        for pi, pot in enumerate(s.potentials):
            if pot["kind"] == "charges":
                I = J = find_group(self.glist, "charges")
                sides = [(I, dens["charges"][1], 1)]
            else:
                I = find_group(self.glist, pot["I"])
                J = find_group(self.glist, pot["J"])
                sides = [(I, dens[self.glist[J][0]][0], 2 if I == J else 1)]
                if I != J:
                    sides.append((J, dens[self.glist[I][0]][0], 1))
            for tgt, rho, mult in sides:
                rk = self._fwd(rho)
                acc = gf.setdefault(tgt, np.zeros((M, Dim), np.float32))
                for d in range(Dim):
                    g = self._inv(self.fk[pi][d] * rk).reshape(M)
                    for _ in range(mult):
                        acc[:, d] += g
        for gi, acc in gf.items():
            name, sites, is_q = self.glist[gi]
            lib.orc32_gather(ctypes.c_int(len(sites)), _p(sites), ctypes.c_int(G), _p(inds), _p(W),
                             ctypes.c_float(np.float32(self.gvol)), _p(np.ascontiguousarray(acc)),
                             _p(self.q) if is_q else None, ctypes.c_int(Dim), _p(f))
        nz = philox_normals(self.seed, self.step_i, self.sites)
        lib.orc32_gjf(ctypes.c_int(len(self.sites)), _p(self.sites), ctypes.c_int(Dim), _p(s.types),
                      _p(s.mass.astype(np.float32)), _p(s.mobility.astype(np.float32)),
                      ctypes.c_float(s.delt), _p(Lr), _p(f), _p(nz), _p(self.x), _p(self.xo),
                      _p(self.old_noise))
        self.step_i += 1


class Trajectory:
    """Runs the reference step order (PS_Box.cu:73-207) with injected noise:
    forces at x_t, then the integrator over its group's sites."""

    def __init__(self, sysm: System, prec=64):
        self.s = sysm
        self.prec = prec
        self.real = np.float32 if prec == 32 else np.float64
        self.x = np.ascontiguousarray(sysm.x, dtype=self.real).reshape(-1).copy()
        self.xo = self.x.copy()                       # ps_integratorGJF.cu:48
        self.old_noise = np.zeros_like(self.x)        # ps_integratorGJF.cu:51
        glist = groups(sysm)
        self.sites = glist[find_group(glist, sysm.integ_group)][1]

    def step(self, unit_noise):
        s, real, lib = self.s, self.real, _lib(self.prec)
        f, _ = forces(s, self.x.reshape(s.N, s.Dim), self.prec)
        f = np.ascontiguousarray(f, dtype=real).reshape(-1)
        un = np.asarray(unit_noise)
        if un.ndim == 2:   # (N, 3) draws: a 2-D box uses the first two of each particle
            un = un[:, :s.Dim]
        nz = np.ascontiguousarray(un, dtype=real).reshape(-1)
        Lr = np.ascontiguousarray(s.L, dtype=real)
        if s.integrator == "GJF":
            getattr(lib, "orc%d_gjf" % self.prec)(
                ctypes.c_int(len(self.sites)), _p(self.sites), ctypes.c_int(s.Dim), _p(s.types),
                _p(s.mass.astype(real)), _p(s.mobility.astype(real)),
                (ctypes.c_float if self.prec == 32 else ctypes.c_double)(s.delt),
                _p(Lr), _p(f), _p(nz), _p(self.x), _p(self.xo), _p(self.old_noise))
        else:
            getattr(lib, "orc%d_em" % self.prec)(
                ctypes.c_int(len(self.sites)), _p(self.sites), ctypes.c_int(s.Dim),
                (ctypes.c_float if self.prec == 32 else ctypes.c_double)(s.delt),
                _p(Lr), _p(f), _p(nz), _p(self.x))
        return f

    def positions(self):
        return self.x.reshape(self.s.N, self.s.Dim)
