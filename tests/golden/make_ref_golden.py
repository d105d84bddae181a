"""Generate golden fixtures from the reference's own CUDA build (run on a GPU machine).

    python tests/golden/make_ref_golden.py --harness oracle/_ref/tild_ref_harness --out DIR

For each system below: write its LAMMPS data file and a current-grammar script (synth),
run the unmodified MATILDA.FT PS_Box through oracle/ref_harness (reference sources built
in place), and pack the inputs plus what the reference computed into DIR/ref_<name>.npz:
  x, types, mol, q, bonds       the input the reference read (after its float parsing)
  inds, W                       d_calcGridWeights tables (first NSTENCIL particles)
  rho_<group>, rhoq             densities after finishInitialization
  f0                            PS_Box::forces() at the initial positions
  energies                      [Ubond, CalcEnergy() of each potential]
  x100                          positions after 100 doTimeStep calls (cuRAND XORWOW noise)
  energies_final                [Ubond, CalcEnergy() of each remaining potential] at the end
  bond_cmd, integrator          the bond and integrator words of the script
Systems with RUNS below execute their script's top-level lines instead (`run nvt N` through
PS_Box::NVT, `modify potential remove i` through PS_Box::modifyBox, main.cu:96-151); they add
  tail                          those lines
  ps_data                       the ps_data.dat the runs wrote (text)
and x100 then holds the positions after the last run.
The committed fixtures under tests/golden/ were produced by this script.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "matilda.ft_b200"))
from tild_b200 import synth  # noqa: E402

NSTENCIL = 256
NSTEPS = 100


def systems():
    return {
        "diblock_o3": synth.small_system(seed=31, order=3),
        "charged_o3": synth.small_system(seed=32, order=3, charges=True, n_free=40),
        "o2": synth.small_system(seed=33, order=2),
        "o4": synth.small_system(seed=34, order=4),
        "o1_oddgrid": synth.small_system(seed=35, order=1, grid=(15, 9, 21), charges=True),
        "erf": synth.small_system(seed=36, order=3, pots=[
            dict(kind="erf2", I="A", J="B", A=0.05, Rp=1.0, sigma=0.5),
            dict(kind="erfG", I="B", J="B", A=0.3, Rp=0.8, sigma=0.5),
            dict(kind="gaussian", I="all", J="A", A=1.5, sigma=0.8)]),
        "c1": synth.config_c1(),
        "angles_o3": synth.small_system(seed=37, order=3, charges=True, angle_params=[
            dict(style="harmonic", k=3.0, theta=120.0), dict(style="wlc", k=2.0)]),
        # harmonic walls (potential wall) beside grid potentials
        "walls_o3": synth.small_system(seed=40, order=3, charges=True, pots=[
            dict(kind="gaussian", I="A", J="B", A=2.0, sigma=0.7), dict(kind="charges", lB=1.0, sigma=0.5),
            dict(kind="wall", I="A", axis="z", pos=2.0, sign=1, k=5.0),
            dict(kind="wall", I="all", axis="x", pos=4.5, sign=-1, k=3.0)]),
        # 2-D boxes (Dim 2): the plane's stencils, k-vectors, noise draws and gvol
        "d2_o3": synth.small_system(seed=38, order=3, charges=True, dim=2, grid=(16, 18, 1)),
        "d2_o4": synth.small_system(seed=39, order=4, dim=2, grid=(15, 12, 1), angle_params=[
            dict(style="harmonic", k=2.0, theta=110.0)]),
        # Euler-Maruyama (ps_integratorEM.cu:39-82: noise sqrt(2 dt), mass and mobility unused)
        "em_o3": synth.small_system(seed=45, order=3, charges=True, integrator="EM"),
        # FENE bonds (ps_deviceBonds.cu:60-62), chains with shorter bonds than r0
        "fene_o3": synth.small_system(seed=42, order=3, bond_rms=0.8, bond_style="fene", bond_k=1.5,
                                      bond_req=2.5),
        # ramped amplitudes (ps_potential.cu:227-248): the table is rescaled to
        # A(t) / Re u(0), which for erf2 and erfG is not A (run through NVT, maxSteps = 100)
        "ramp_o3": synth.small_system(seed=43, order=3, pots=[
            dict(kind="erf2", I="A", J="B", A=0.05, Rp=1.0, sigma=0.5, ramp=0.4),
            dict(kind="erfG", I="B", J="B", A=0.3, Rp=0.8, sigma=0.5, ramp=0.05),
            dict(kind="gaussian", I="A", J="A", A=1.0, sigma=0.7, ramp=3.0)]),
        # modify potential remove between two runs (PS_Box.cu:848-870)
        "modify_o3": synth.small_system(seed=44, order=3, charges=True),
    }


# systems whose script's top-level lines run (main.cu:96-151) instead of NSTEPS doTimeStep calls
RUNS = {
    "ramp_o3": ["run nvt %d" % NSTEPS],
    "modify_o3": ["run nvt 40", "modify potential remove 1", "run nvt 60"],
}


def read_data_positions(path, n, dim, charges):
    """x as the reference parsed it (fscanf %f -> float32)."""
    lines = open(path).read().splitlines()
    k = lines.index("Atoms") + 2
    x = np.zeros((n, dim), np.float32)
    for i in range(n):
        w = lines[k + i].split()
        idx = int(w[0]) - 1
        c = 4 if charges else 3
        x[idx] = np.array(w[c:c + dim], dtype=np.float32)
    return x


def run(harness, name, spec, out, time_steps=0):
    with tempfile.TemporaryDirectory() as d:
        tail = RUNS.get(name)
        spec.log_freq = 1000000 if tail is None else 10
        scr, data = spec.write(d, steps=NSTEPS, tail=tail)
        dump = os.path.join(d, "dump")
        os.makedirs(dump)
        cmd = [os.path.abspath(harness), os.path.basename(scr), dump, str(NSTEPS), str(time_steps)]
        if tail is not None:
            cmd.append("script")
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=1800)
        if r.returncode != 0:
            raise RuntimeError("%s: harness failed rc=%d\n%s" % (name, r.returncode, r.stderr[-2000:]))
        meta = {}
        groups = []
        for line in open(os.path.join(dump, "meta.txt")):
            k, v = line.split(None, 1)
            if k == "group":
                groups.append(v.strip())
            else:
                meta[k] = v.strip()
        N, D, G, M = (int(meta[k]) for k in ("N", "Dim", "G", "M"))
        ld = lambda f, t: np.fromfile(os.path.join(dump, f), dtype=t)  # noqa: E731
        res = dict(
            x=read_data_positions(data, N, D, spec.charges is not None), types=spec.types, mol=spec.mol,
            bonds=spec.bonds.astype(np.int32), L=spec.L, grid=spec.grid, order=np.int32(spec.order),
            seed=np.int64(spec.seed), delt=np.float32(spec.delt),
            inds=ld("gridInds.i32", np.int32).reshape(N, G)[:NSTENCIL],
            W=ld("gridW.f32", np.float32).reshape(N, G)[:NSTENCIL],
            f0=ld("f0.f32", np.float32).reshape(N, D), energies=ld("energies.f64", np.float64),
            x100=ld("x_final.f32", np.float32).reshape(N, D), gvol=np.float64(meta["gvol"]),
            energies_final=ld("energies_final.f64", np.float64), bond_cmd=np.array(spec.bond_command()),
            integrator=np.array(spec.integrator),
            groups=np.array(groups), cuda_error=np.array(meta.get("cuda_error", "")))
        if tail is not None:
            res["tail"] = np.array(tail)
            res["ps_data"] = np.array(open(os.path.join(d, "ps_data.dat")).read())
        if spec.charges is not None:
            res["q"] = spec.charges
            res["rhoq"] = ld("rhoq_charges.f32", np.float32)
        for g in groups:
            res["rho_" + g] = ld("rho_%s.f32" % g, np.float32)
        res["potentials"] = np.array([repr(p) for p in spec.potentials])
        if len(spec.angles):
            res["angles"] = spec.angles.astype(np.int32)
            res["angle_types"] = spec.angle_types.astype(np.int32)
            res["angle_params"] = np.array([repr(a) for a in spec.angle_params])
            res["uangle"] = ld("uangle.f64", np.float64)
        np.savez_compressed(os.path.join(out, "ref_%s.npz" % name), **res)
        return meta.get("ms_per_step")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--harness", default=os.path.join(ROOT, "oracle", "_ref", "tild_ref_harness"))
    ap.add_argument("--out", required=True)
    ap.add_argument("--time", action="store_true", help="also time the reference on C1 and C2")
    ap.add_argument("--only", nargs="*", help="generate only these systems")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for name, spec in systems().items():
        if a.only and name not in a.only:
            continue
        ms = run(a.harness, name, spec, a.out, time_steps=200 if (a.time and name == "c1") else 0)
        print(name, "ok", "" if ms is None else "ms_per_step %s" % ms, flush=True)
    if a.time:
        spec = synth.config_c2()
        with tempfile.TemporaryDirectory() as d:
            spec.log_freq = 1000000
            scr, _ = spec.write(d, steps=0)
            dump = os.path.join(d, "dump")
            os.makedirs(dump)
            r = subprocess.run([os.path.abspath(a.harness), os.path.basename(scr), dump, "2", "20"], cwd=d,
                               capture_output=True, text=True, timeout=3000)
            print("c2", "rc", r.returncode, [l for l in r.stdout.splitlines() if l.startswith("ms_per_step")],
                  flush=True)


if __name__ == "__main__":
    main()
