"""Generate the run-output fixture from the reference's own CUDA build (run on a GPU
machine with oracle/ref_harness built).

    python tests/golden/make_ref_outputs.py --out DIR

Writes OUTPUT_SYSTEM's LAMMPS data file and its script with the output words below, runs
the unmodified reference through oracle/ref_harness in NVT mode (PS_Box::NVT for NSTEPS
steps: per-step outputs at the script's frequencies plus the run's closing outputs), and
packs into DIR/outputs_ref.npz:
  script, data                  the inputs (text)
  nsteps                        steps run
  traj                          traj.lammpstrj (text; PS_Box::writeLammpsTraj)
  gsd                           traj.gsd (bytes; PS_Box::writeGSDtraj)
  density_<group>               density-<group>.bin (bytes; writeFields)
  ps_data, final_data           ps_data.dat and final.input.data (text)
The committed tests/golden/outputs_ref.npz was produced by this script.
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

NSTEPS = 12
# lammpstrj every 3 steps; fields at 0, 2, then the interval doubling after each frame
# (logspace 2.0); GSD every 5 steps; thermo every 4 steps
OUTPUT_WORDS = ["trajFreq 3", "fieldFreq 2 logspace 2.0", "gsdFreq 5", "logFreq 4"]


def output_system():
    s = synth.small_system(seed=41, order=3, charges=True,
                           angle_params=[dict(style="harmonic", k=3.0, theta=120.0)])
    s.name = "outputs"
    return s


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--harness", default=os.path.join(ROOT, "oracle", "_ref", "tild_ref_harness"))
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    s = output_system()
    with tempfile.TemporaryDirectory() as d:
        scr, data = s.write(d, steps=NSTEPS, extra=OUTPUT_WORDS)
        dump = os.path.join(d, "dump")
        os.makedirs(dump)
        r = subprocess.run([os.path.abspath(a.harness), os.path.basename(scr), dump, str(NSTEPS), "0", "nvt"],
                           cwd=d, capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError("harness failed rc=%d\n%s\n%s" % (r.returncode, r.stdout[-3000:], r.stderr[-2000:]))
        out = {"script": np.array(open(scr).read()), "data": np.array(open(data).read()),
               "nsteps": np.array(NSTEPS),
               "traj": np.array(open(os.path.join(d, "traj.lammpstrj")).read()),
               "gsd": np.frombuffer(open(os.path.join(d, "traj.gsd"), "rb").read(), np.uint8),
               "ps_data": np.array(open(os.path.join(d, "ps_data.dat")).read()),
               "final_data": np.array(open(os.path.join(d, "final.input.data")).read())}
        for f in sorted(os.listdir(d)):
            if f.startswith("density-") and f.endswith(".bin"):
                out["density_" + f[len("density-"):-4]] = np.frombuffer(open(os.path.join(d, f), "rb").read(),
                                                                         np.uint8)
    np.savez_compressed(os.path.join(a.out, "outputs_ref.npz"), **out)
    print("outputs ok", sorted(out), flush=True)


if __name__ == "__main__":
    main()
