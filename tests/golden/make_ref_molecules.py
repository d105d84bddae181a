"""Generate the molecule-builder fixture from the reference's own CUDA build (run on a GPU
machine with oracle/ref_harness built).

    python tests/golden/make_ref_molecules.py --out DIR

Runs the unmodified reference on MOLECULE_SCRIPT (below; the same text is used by the
tests) through oracle/ref_harness with zero steps, and packs into DIR/molecules_ref.npz:
  x0                          d_x after set-up (the positions makeLinear produced)
  init_data                   the reference's init.input.data (writeDataConfig), as text
The committed tests/golden/molecules_ref.npz was produced by this script.
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

# two `molecule linear` commands: charged AB diblocks with per-block bond and angle types
# (nmolecs), then B homopolymers with angles (phi); positions come from the host RNG
MOLECULE_SCRIPT = """box ps
Dim 3
boxLengths 10.0 11.0 9.0
grid 20 22 18
pmeorder 3
randSeed 1234
rho0 3.0
species A mass 1.0 mobility 1.0
species B mass 1.0 mobility 1.0
molecule linear nmolecs 30 2 8 A 8 B charge 1 -1 bondType 1 2 angleType 1 0
molecule linear phi 0.2 1 12 B angleType 2 charge 0.0
bond 1 harmonic 1.5 0.0
bond 2 harmonic 2.0 0.5
angle 1 harmonic 2.0 120.0
angle 2 wlc 1.0
potential gaussian A B 2.0 0.7
potential charges 1.0 0.5
integrator all GJF delt 0.005
endBox
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--harness", default=os.path.join(ROOT, "oracle", "_ref", "tild_ref_harness"))
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as d:
        with open(os.path.join(d, "input"), "w") as fh:
            fh.write(MOLECULE_SCRIPT)
        dump = os.path.join(d, "dump")
        os.makedirs(dump)
        r = subprocess.run([os.path.abspath(a.harness), "input", dump, "0"], cwd=d, capture_output=True, text=True,
                           timeout=600)
        if r.returncode != 0:
            raise RuntimeError("harness failed rc=%d\n%s\n%s" % (r.returncode, r.stdout[-3000:], r.stderr[-2000:]))
        meta = dict(line.split(None, 1) for line in open(os.path.join(dump, "meta.txt")) if not line.startswith("group"))
        N, D = int(meta["N"]), int(meta["Dim"])
        x0 = np.fromfile(os.path.join(dump, "x_final.f32"), dtype=np.float32).reshape(N, D)
        init = open(os.path.join(d, "init.input.data")).read()
    np.savez_compressed(os.path.join(a.out, "molecules_ref.npz"), x0=x0, init_data=np.array(init))
    print("molecules ok", N, flush=True)


if __name__ == "__main__":
    main()
