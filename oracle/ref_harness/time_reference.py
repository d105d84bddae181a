"""Time the reference's own CUDA build in its plain per-job form on the batched (C3) and
served (C5) workloads: one harness process per job, jobs one after another (run on a GPU
machine with the harness built by oracle/ref_harness/Makefile).

    python oracle/ref_harness/time_reference.py [--harness oracle/_ref/tild_ref_harness]

For each job the synthetic system is written as a LAMMPS data file plus a script in the
reference's grammar, and the unmodified reference runs it through the harness: set-up,
one step, then `time_steps` steps timed with CUDA events (ms_per_step).  The job's plain
per-job time is its process wall time minus the timed steps plus `steps` x ms_per_step
(the set-up counted once, as a `matilda.ft -in job.in` run would).  Prints one JSON line
per workload.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "matilda.ft_b200"))
from tild_b200 import synth  # noqa: E402


def time_job(harness, spec, steps, time_steps):
    with tempfile.TemporaryDirectory() as d:
        spec.log_freq = 1000000
        scr, _ = spec.write(d, steps=0)
        dump = os.path.join(d, "dump")
        os.makedirs(dump)
        t0 = time.perf_counter()
        r = subprocess.run([os.path.abspath(harness), os.path.basename(scr), dump, "1", str(time_steps)], cwd=d,
                           capture_output=True, text=True, timeout=1800)
        wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError("harness failed rc=%d\n%s" % (r.returncode, r.stderr[-2000:]))
    ms = [float(line.split()[1]) for line in r.stdout.splitlines() if line.startswith("ms_per_step")][0]
    job_s = wall - time_steps * ms * 1e-3 + steps * ms * 1e-3
    return ms, job_s


def summarize(name, rows):
    work = sum(n * s for n, s, _, _ in rows)
    return {"workload": name, "jobs": len(rows), "particle_steps": work,
            "plain_per_job_value": work / sum(j for _, _, _, j in rows),
            "steady_state_value": work / sum(s * ms * 1e-3 for _, s, ms, _ in rows),
            "unit": "particle-steps/s"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--harness", default=os.path.join(ROOT, "oracle", "_ref", "tild_ref_harness"))
    ap.add_argument("--c3-replicas", type=int, default=64)
    ap.add_argument("--c3-steps", type=int, default=500)
    ap.add_argument("--c5-jobs", type=int, default=40)
    ap.add_argument("--time-steps", type=int, default=30)
    a = ap.parse_args()
    rows = []
    for spec in synth.config_c3(replicas=a.c3_replicas):
        ms, job = time_job(a.harness, spec, a.c3_steps, a.time_steps)
        rows.append((spec.N, a.c3_steps, ms, job))
    print(json.dumps(summarize("c3: %d diblock replicas, %d steps each" % (a.c3_replicas, a.c3_steps), rows)),
          flush=True)
    rows = []
    for spec, steps in synth.config_c5_jobs(njobs=a.c5_jobs):
        ms, job = time_job(a.harness, spec, steps, a.time_steps)
        rows.append((spec.N, steps, ms, job))
    print(json.dumps(summarize("c5: %d jobs" % a.c5_jobs, rows)), flush=True)


if __name__ == "__main__":
    main()
