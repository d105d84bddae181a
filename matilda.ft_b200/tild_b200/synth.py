"""Seeded synthetic TILD systems and their MATILDA.FT input files.

Writes LAMMPS-style data files in the layout that MATILDA.FT's ``writeDataConfig``
emits and ``readDataConfig`` reads (PS_Box.cu:629-748, PS_Box_initialization.cu:787-997),
and ``box ps ... endBox`` scripts in the current grammar (PS_Box_initialization.cu:68-339,
main.cu:96-151).  No public benchmark data is involved: every system is drawn from a
numpy ``default_rng(seed)`` with the shapes of the benchmark workloads.
"""
from __future__ import annotations

import math
import os

import numpy as np

SIGMA_GAUSS = 0.7071  # sqrt(2) * a for smearing a = 0.5 (pair kernel of two Gaussians)


def random_walk_chains(rng, nchains, nper, L, bond_rms=1.0):
    """First bead uniform in [0, L)^3; each next bead = previous + N(0, bond_rms^2/3)
    per axis; wrapped into [0, L)."""
    L = np.asarray(L, np.float64)
    first = rng.uniform(0.0, 1.0, size=(nchains, 1, 3)) * L
    steps = rng.normal(0.0, bond_rms / math.sqrt(3.0), size=(nchains, nper - 1, 3))
    pos = np.concatenate([first, first + np.cumsum(steps, axis=1)], axis=1)
    return np.mod(pos, L).reshape(-1, 3)


def chain_bonds(nchains, nper, offset=0):
    base = offset + np.arange(nchains)[:, None] * nper
    i = (base + np.arange(nper - 1)[None, :]).reshape(-1)
    return np.stack([i, i + 1], axis=1)


def potential_command(p):
    """Script line of one potential spec (dict with kind and its parameters)."""
    k = p["kind"]
    ramp = (" ramp %.9g" % p["ramp"]) if "ramp" in p else ""
    if k == "gaussian":
        return "potential gaussian %s %s %.9g %.9g" % (p["I"], p["J"], p["A"], p["sigma"]) + ramp
    if k in ("erf2", "erfG"):
        return "potential %s %s %s %.9g %.9g %.9g" % (k, p["I"], p["J"], p["A"], p["Rp"], p["sigma"]) + ramp
    if k == "charges":
        return "potential charges %.9g %.9g" % (p["lB"], p["sigma"])
    if k == "wall":   # potential wall <group> <axis> <position> <side +1|-1> <k>
        return "potential wall %s %s %.9g %d %.9g" % (p["I"], p["axis"], p["pos"], p["sign"], p["k"])
    raise ValueError("unknown potential kind " + k)


class SystemSpec:
    """Arrays + script parameters of one synthetic box."""

    def __init__(self, name, L, grid, x, types, species, bonds, mol, charges=None,
                 potentials=(), order=3, delt=0.005, bond_k=1.5, bond_req=0.0, seed=1,
                 dim=3, integrator="GJF", masses=None, mobility=None, log_freq=100, angles=None,
                 angle_types=None, angle_params=(), bond_style="harmonic", max_bonds=None):
        self.name = name
        self.L = np.asarray(L, np.float32)
        self.grid = np.asarray(grid, np.int32)
        self.x = np.asarray(x, np.float32)
        self.types = np.asarray(types, np.int32)
        self.species = list(species)
        self.bonds = np.asarray(bonds, np.int64).reshape(-1, 2)
        self.mol = np.asarray(mol, np.int32)
        self.charges = None if charges is None else np.asarray(charges, np.float32)
        self.potentials = list(potentials)
        self.order = order
        self.delt = delt
        self.bond_k = bond_k
        self.bond_req = bond_req
        self.bond_style = bond_style   # "harmonic" or "fene" (ps_deviceBonds.cu:54-62)
        self.max_bonds = max_bonds     # MAXBONDS word (None: the reference's default of 2)
        self.seed = seed
        self.dim = dim
        self.integrator = integrator
        self.masses = masses or [1.0] * len(self.species)
        self.mobility = mobility or [1.0] * len(self.species)
        self.log_freq = log_freq
        # angles (i, middle j, k), 0-based types, and per type dict(style="harmonic"|"wlc",
        # k=..., theta=degrees)
        self.angles = np.zeros((0, 3), np.int64) if angles is None else np.asarray(angles, np.int64).reshape(-1, 3)
        self.angle_types = (np.zeros(len(self.angles), np.int32) if angle_types is None
                            else np.asarray(angle_types, np.int32))
        self.angle_params = list(angle_params)

    def angle_commands(self):
        out = []
        for t, a in enumerate(self.angle_params):
            if a["style"] == "harmonic":
                out.append("angle %d harmonic %.9g %.9g" % (t + 1, a["k"], a["theta"]))
            else:
                out.append("angle %d wlc %.9g" % (t + 1, a["k"]))
        return out

    @property
    def N(self):
        return self.x.shape[0]

    @property
    def M(self):
        return int(np.prod(self.grid))

    # -- files -----------------------------------------------------------------------
    def write_data(self, path):
        """LAMMPS data file, writeDataConfig layout (PS_Box.cu:629-748)."""
        N, D = self.N, self.dim
        nbt = 1 if len(self.bonds) else 0
        lines = ["Created by tild-b200 synth", "",
                 "%d atoms" % N, "%d bonds" % len(self.bonds), "%d angles" % len(self.angles), "",
                 "%d atom types" % len(self.species), "%d bond types" % nbt,
                 "%d angle types" % len(self.angle_params), "",
                 "0.0 %.9g xlo xhi" % self.L[0], "0.0 %.9g ylo yhi" % self.L[1],
                 ("0.0 %.9g zlo zhi" % self.L[2]) if D > 2 else "0.0 1.0 zlo zhi", "",
                 "Masses", ""]
        for t, m in enumerate(self.masses):
            lines.append("%d %.9g" % (t + 1, m))
        lines += ["", "Atoms", ""]
        body = []
        ids = np.arange(1, N + 1)
        cols = [ids, self.mol + 1, self.types + 1]
        fmt = ["%d", "%d", "%d"]
        if self.charges is not None:
            cols.append(self.charges)
            fmt.append("%.6g")
        for d in range(D):
            cols.append(self.x[:, d])
            fmt.append("%.9g")
        if D < 3:
            cols.append(np.zeros(N))
            fmt.append("%.1f")
        arr = np.empty((N, len(cols)), dtype=object)
        with open(path, "w") as fh:
            fh.write("\n".join(lines) + "\n")
            tbl = np.column_stack([np.asarray(c, np.float64) for c in cols])
            np.savetxt(fh, tbl, fmt=" ".join(fmt))
            fh.write("\nBonds\n\n")
            if len(self.bonds):
                b = np.column_stack([np.arange(1, len(self.bonds) + 1), np.ones(len(self.bonds)),
                                     self.bonds[:, 0] + 1, self.bonds[:, 1] + 1]).astype(np.int64)
                np.savetxt(fh, b, fmt="%d %d %d %d")
            if len(self.angles):
                fh.write("\nAngles\n\n")
                a = np.column_stack([np.arange(1, len(self.angles) + 1), self.angle_types + 1,
                                     self.angles + 1]).astype(np.int64)
                np.savetxt(fh, a, fmt="%d %d %d %d %d")
            fh.write("\n")
        del arr, body

    def bond_command(self):
        return "bond 1 %s %.9g %.9g" % (self.bond_style, self.bond_k, self.bond_req)

    def script(self, data_name, steps=100, extra=(), tail=None):
        """Current-grammar input script (PS_Box_initialization.cu:68-339).  After endBox:
        `run nvt <steps>`, or the top-level lines ``tail`` (run / modify, main.cu:96-151)."""
        D = self.dim
        s = ["box ps", "Dim %d" % D,
             "boxLengths " + " ".join("%.9g" % v for v in self.L[:D]),
             "grid " + " ".join(str(int(v)) for v in self.grid[:D]),
             "pmeorder %d" % self.order, "randSeed %d" % self.seed]
        if self.charges is not None:
            s.append("doCharges")
        if self.max_bonds:
            s.append("MAXBONDS %d" % self.max_bonds)
        for t, lb in enumerate(self.species):
            s.append("species %s mass %.9g mobility %.9g" % (lb, self.masses[t], self.mobility[t]))
        s.append("readData %s" % data_name)
        if len(self.bonds):
            s.append(self.bond_command())
        s += self.angle_commands()
        s += [potential_command(p) for p in self.potentials]
        s.append("integrator all %s delt %.9g" % (self.integrator, self.delt))
        s.append("logFreq %d" % self.log_freq)
        s += list(extra)
        s.append("endBox")
        s += ["run nvt %d" % steps] if tail is None else list(tail)
        return "\n".join(s) + "\n"

    def write(self, directory, steps=100, extra=(), tail=None):
        os.makedirs(directory, exist_ok=True)
        data = os.path.join(directory, self.name + ".data")
        self.write_data(data)
        scr = os.path.join(directory, self.name + ".in")
        with open(scr, "w") as fh:
            fh.write(self.script(os.path.basename(data), steps, extra, tail))
        return scr, data

    # -- compact partner lists (both directions, like readDataConfig :897-926) ------
    def partner_lists(self, maxb=None):
        N = self.N
        deg = np.zeros(N, np.int32)
        np.add.at(deg, self.bonds[:, 0], 1)
        np.add.at(deg, self.bonds[:, 1], 1)
        mb = int(deg.max()) if len(self.bonds) else 0
        maxb = max(mb, maxb or 2)
        partner = np.zeros((N, maxb), np.int32)
        btype = np.zeros((N, maxb), np.int32)
        nb = np.zeros(N, np.int32)
        for a, b in self.bonds:
            i1, i2 = (a, b) if a < b else (b, a)
            partner[i1, nb[i1]] = i2; nb[i1] += 1
            partner[i2, nb[i2]] = i1; nb[i2] += 1
        return nb, partner, btype


def diblock_melt(nchains, nper, L, grid, chi=1.0, rho0=4.88, kappa=25.0, fA=0.5, seed=1,
                 order=3, name="diblock", sigma=SIGMA_GAUSS, extra_pots=()):
    rng = np.random.default_rng(seed)
    x = random_walk_chains(rng, nchains, nper, [L, L, L])
    nA = int(round(fA * nper))
    types = np.tile(np.r_[np.zeros(nA, np.int32), np.ones(nper - nA, np.int32)], nchains)
    mol = np.repeat(np.arange(nchains, dtype=np.int32), nper)
    aa = kappa / rho0
    ab = (kappa + chi) / rho0
    pots = [dict(kind="gaussian", I="A", J="A", A=aa, sigma=sigma),
            dict(kind="gaussian", I="B", J="B", A=aa, sigma=sigma),
            dict(kind="gaussian", I="A", J="B", A=ab, sigma=sigma)] + list(extra_pots)
    return SystemSpec(name, [L, L, L], [grid] * 3, x, types, ["A", "B"],
                      chain_bonds(nchains, nper), mol, potentials=pots, order=order, seed=seed)


def config_c1(seed=1):
    """1,000 AB diblocks of N=20 (10 A + 10 B), L=16, 32^3 grid, kappa/rho0=25/4.88,
    chi=1, GJF dt=0.005."""
    return diblock_melt(1000, 20, 16.0, 32, chi=1.0, rho0=4.88, seed=seed, name="c1_diblock")


def config_c2(seed=2, scale=1.0):
    """Polyelectrolyte coacervate: 8,000 + 8,000 chains of N=32 (q=+1/-1), 256,000 +
    256,000 counterions, neutral solvent to 2,097,152 particles, rho0=5, 192^3 grid.
    ``scale`` shrinks particle counts (and L, grid) for tests."""
    rng = np.random.default_rng(seed)
    nch = int(round(8000 * scale))
    nper = 32
    npoly = 2 * nch * nper
    nci = nch * nper
    ntot = int(round(2097152 * scale))
    nsolv = ntot - npoly - 2 * nci
    L = (ntot / 5.0) ** (1.0 / 3.0)
    grid = max(8, int(round(192 * scale ** (1.0 / 3.0))))
    xp = random_walk_chains(rng, 2 * nch, nper, [L, L, L])
    xr = rng.uniform(0.0, L, size=(2 * nci + nsolv, 3))
    x = np.concatenate([xp, xr]).astype(np.float32)
    q = np.concatenate([np.ones(nch * nper), -np.ones(nch * nper),
                        -np.ones(nci), np.ones(nci), np.zeros(nsolv)]).astype(np.float32)
    types = np.concatenate([np.zeros(npoly), np.ones(2 * nci), 2 * np.ones(nsolv)]).astype(np.int32)
    mol = np.concatenate([np.repeat(np.arange(2 * nch), nper),
                          2 * nch + np.arange(2 * nci + nsolv)]).astype(np.int32)
    pots = [dict(kind="gaussian", I="all", J="all", A=25.0 / 5.0, sigma=SIGMA_GAUSS),
            dict(kind="charges", lB=1.0, sigma=0.5)]
    return SystemSpec("c2_coacervate", [L, L, L], [grid] * 3, x, types, ["P", "C", "S"],
                      chain_bonds(2 * nch, nper), mol, charges=q, potentials=pots, order=3,
                      seed=seed)


def config_c4(seed=4, scale=1.0):
    """1,048,576-particle diblock melt (N=32, fA=0.5, chi=1.5, rho0=5), 160^3 grid,
    Gaussian + erf2 (Rp=1.0, sigma=0.5)."""
    nch = int(round(32768 * scale))
    ntot = nch * 32
    L = (ntot / 5.0) ** (1.0 / 3.0)
    grid = max(8, int(round(160 * scale ** (1.0 / 3.0))))
    erf = [dict(kind="erf2", I="A", J="B", A=0.01, Rp=1.0, sigma=0.5)]
    return diblock_melt(nch, 32, L, grid, chi=1.5, rho0=5.0, seed=seed, name="c4_precision",
                        extra_pots=erf)


def smooth_grid(n):
    """Nearest integer >= 8 to n whose prime factors are 2, 3, 5, 7."""
    def smooth(m):
        for f in (2, 3, 5, 7):
            while m % f == 0:
                m //= f
        return m == 1
    best = None
    for d in range(0, 64):
        for m in (int(round(n)) - d, int(round(n)) + d):
            if m >= 8 and smooth(m):
                best = m if best is None or abs(m - n) < abs(best - n) else best
        if best is not None:
            return best
    return max(8, int(round(n)))


def config_c3(seed=3, replicas=64, nmin=1.0e4, nmax=4.0e5):
    """Uneven AB diblock replicas: chain length in {16, 24, 32, 48}, particle count
    log-uniform in [nmin, nmax] rounded to whole chains, rho0 = 5, grid spacing ~0.4 on a
    2,3,5,7-smooth grid (the last replica takes a prime grid size), chi ~ U[0.2, 2.0],
    A fraction ~ U[0.2, 0.8].  Replica r draws from seed + r."""
    out = []
    for r in range(replicas):
        rng = np.random.default_rng(seed + r)
        nper = int(rng.choice([16, 24, 32, 48]))
        ntot = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        nch = max(1, int(round(ntot / nper)))
        L = (nch * nper / 5.0) ** (1.0 / 3.0)
        grid = smooth_grid(L / 0.4)
        if r == replicas - 1:   # a prime size exercises the generic radix
            grid = next(p for p in range(int(L / 0.4) | 1, 10000, 2) if all(p % k for k in range(3, int(p ** 0.5) + 1, 2)))
        chi = float(rng.uniform(0.2, 2.0))
        fA = float(rng.uniform(0.2, 0.8))
        out.append(diblock_melt(nch, nper, L, grid, chi=chi, rho0=5.0, fA=fA, seed=seed + r,
                                name="c3_replica%d" % r))
    return out


def config_c5_jobs(seed=5, njobs=40, nmin=2.0e4, nmax=2.0e5, smin=100, smax=400):
    """Served jobs: diblock melts or coacervates (equal odds), particle count log-uniform
    in [nmin, nmax], steps uniform in [smin, smax].  Returns (spec, steps) pairs; job j
    draws from seed + j."""
    jobs = []
    for j in range(njobs):
        rng = np.random.default_rng(seed + j)
        ntot = float(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        steps = int(rng.integers(smin, smax + 1))
        if rng.uniform() < 0.5:
            nper = 32
            nch = max(1, int(round(ntot / nper)))
            L = (nch * nper / 5.0) ** (1.0 / 3.0)
            spec = diblock_melt(nch, nper, L, smooth_grid(L / 0.4), chi=float(rng.uniform(0.2, 2.0)), rho0=5.0,
                                seed=seed + j, name="c5_diblock%d" % j)
        else:
            spec = config_c2(seed=seed + j, scale=ntot / 2097152.0)
            spec.name = "c5_coacervate%d" % j
            g = smooth_grid(float(spec.L[0]) / 0.4)
            spec.grid = [g, g, g]
        jobs.append((spec, steps))
    return jobs


def chain_angles(nchains, nper, offset=0):
    """(i-1, i, i+1) triples along every chain."""
    out = []
    for c in range(nchains):
        b = offset + c * nper
        out += [(b + i - 1, b + i, b + i + 1) for i in range(1, nper - 1)]
    return np.array(out, np.int64).reshape(-1, 3)


def small_system(seed=0, n_chains=20, nper=8, L=6.0, grid=(12, 12, 12), order=3, charges=False,
                 dim=3, pots=None, n_free=0, angle_params=None, bond_rms=1.0, **spec_kw):
    """A tiny randomised system for oracle comparisons.  spec_kw go to SystemSpec
    (integrator, bond_style, bond_k, bond_req, ...)."""
    rng = np.random.default_rng(seed)
    Lv = np.array([L, L * 1.1, L * 0.9][:dim] + [1.0] * (3 - dim))
    if dim == 3:
        x = random_walk_chains(rng, n_chains, nper, Lv, bond_rms)
    else:
        x3 = random_walk_chains(rng, n_chains, nper, np.r_[Lv[:2], 1.0], bond_rms)
        x = x3
    if n_free:
        x = np.concatenate([x, rng.uniform(0, 1, size=(n_free, 3)) * Lv])
    N = x.shape[0]
    types = rng.integers(0, 2, size=N).astype(np.int32)
    mol = np.r_[np.repeat(np.arange(n_chains), nper), n_chains + np.arange(n_free)].astype(np.int32)
    q = None
    if charges:
        q = rng.choice([-1.0, 0.0, 1.0], size=N).astype(np.float32)
        s = q.sum()
        idx = np.nonzero(q == (1.0 if s > 0 else -1.0))[0]
        q[idx[: int(abs(s))]] = 0.0
    if pots is None:
        pots = [dict(kind="gaussian", I="A", J="A", A=2.0, sigma=0.7),
                dict(kind="gaussian", I="A", J="B", A=3.0, sigma=0.7)]
        if charges:
            pots.append(dict(kind="charges", lB=1.0, sigma=0.5))
    grid = list(grid)[:dim] + [1] * (3 - dim)
    ang, atyp = None, None
    if angle_params:   # chain triples, types alternating over the given angle types
        ang = chain_angles(n_chains, nper)
        atyp = (np.arange(len(ang)) % len(angle_params)).astype(np.int32)
    return SystemSpec("small%d" % seed, Lv, grid, x[:, :dim] if dim == 2 else x, types, ["A", "B"],
                      chain_bonds(n_chains, nper), mol, charges=q, potentials=pots, order=order,
                      seed=seed + 11, dim=dim, angles=ang, angle_types=atyp,
                      angle_params=angle_params or (), **spec_kw)


def branched_system(seed=0, L=7.0, grid=(14, 14, 14), order=3, charges=True):
    """Branched molecules for the bond list: combs (a 12-bead backbone with 3-bead side
    chains on beads 2, 6 and 10: degree 3) and stars (a centre with five 4-bead arms:
    degree 5), plus free beads; MAXBONDS 5."""
    rng = np.random.default_rng(seed)
    xs, bonds, mol = [], [], []
    def walk(start, n):
        pts = [start]
        for _ in range(n - 1):
            pts.append(pts[-1] + rng.normal(0.0, 1.0 / math.sqrt(3.0), 3))
        return pts
    n = 0
    for c in range(6):   # combs
        back = walk(rng.uniform(0, L, 3), 12)
        ids = list(range(n, n + 12))
        xs += back
        bonds += [(ids[i], ids[i + 1]) for i in range(11)]
        mol += [c] * 12
        n += 12
        for b in (2, 6, 10):
            side = walk(back[b] + rng.normal(0.0, 0.6, 3), 3)
            xs += side
            bonds += [(ids[b], n)] + [(n + i, n + i + 1) for i in range(2)]
            mol += [c] * 3
            n += 3
    for s_ in range(5):   # stars
        centre = rng.uniform(0, L, 3)
        xs.append(centre)
        c0 = n
        mol.append(6 + s_)
        n += 1
        for a in range(5):
            arm = walk(centre + rng.normal(0.0, 0.6, 3), 4)
            xs += arm
            bonds += [(c0, n)] + [(n + i, n + i + 1) for i in range(3)]
            mol += [6 + s_] * 4
            n += 4
    for f in range(30):   # free beads
        xs.append(rng.uniform(0, L, 3))
        mol.append(11 + f)
        n += 1
    x = np.mod(np.array(xs), L)
    N = x.shape[0]
    types = rng.integers(0, 2, size=N).astype(np.int32)
    q = None
    if charges:
        q = rng.choice([-1.0, 0.0, 1.0], size=N).astype(np.float32)
        s = q.sum()
        idx = np.nonzero(q == (1.0 if s > 0 else -1.0))[0]
        q[idx[: int(abs(s))]] = 0.0
    pots = [dict(kind="gaussian", I="A", J="B", A=2.5, sigma=0.7),
            dict(kind="gaussian", I="all", J="all", A=1.0, sigma=0.7)]
    if charges:
        pots.append(dict(kind="charges", lB=1.0, sigma=0.5))
    return SystemSpec("branched%d" % seed, [L, L, L], list(grid), x, types, ["A", "B"], np.array(bonds), mol,
                      charges=q, potentials=pots, order=order, seed=seed + 11, max_bonds=5)
