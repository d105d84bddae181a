"""Benchmark of the B200 TILD step (particle-steps/s) on the coacervate workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one per GPU; N > 1 runs independent replicas, one per rank -- the step does
not shard): polyelectrolyte coacervate, 2,097,152 particles (8,000 + 8,000 chains of
N=32, q = +1/-1, 512,000 counterions, neutral solvent), rho0 = 5, L = 74.85, 192^3 grid,
pmeorder 3, `potential gaussian all all 5.0 0.7071` + `potential charges 1.0 0.5`,
harmonic bonds k = 1.5, GJF dt = 0.005, Philox noise.  Synthetic data (numpy seed 2).

value: particle-steps/s of K graph-replayed steps with all state resident in HBM, timed
with CUDA events on the box's stream, max over ranks.  The per-step working set
(about 0.8 GB of grids and particle arrays) is larger than the 126 MB L2, so no flush
is needed between steps.
e2e: the same metric through the C ABI for one job of S steps: positions uploaded from
pinned host memory, S steps, positions read back; copies inside the timed region.
batched: C3, 64 uneven diblock replicas stepped as one batch (every stage of a step one
kernel launch over all replicas), beside the same jobs one after another and in the job
pool.  served: C5, a Poisson job stream through the job pool, with p50/p99 latency.
--impl reference: MATILDA.FT's own CUDA build (the unmodified sources compiled into
oracle/_ref by oracle/ref_harness/Makefile) on the same workload, GPU and metric, rank 0
only, plus its plain per-job form on samples of the batched and served job lists; when
that build is absent, the reference's step restated on the host cores (oracle CpuStep).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "matilda.ft_b200"))

import numpy as np  # noqa: E402

METRIC = "particle-steps/s"
WORKLOAD = ("c2_coacervate: 2,097,152 particles, 192^3 grid, pmeorder 3, gaussian(all,all) + "
            "smeared charges (lB 1.0, sigma 0.5), harmonic bonds, GJF dt 0.005")
STAGES = ["deposit", "fft_x_fwd", "fft_y_fwd", "kspace_z", "fft_y_inv", "fft_x_inv", "gather", "integrate"]
KERNEL_NAMES = {"deposit": "k_deposit", "fft_x_fwd": "k_xfwd", "fft_y_fwd": "k_ypass<false>",
                "kspace_z": "k_kspace_z", "fft_y_inv": "k_ypass<true>", "fft_x_inv": "k_xinv",
                "gather": "k_gather_paired", "integrate": "k_integrate"}
KERNELS_PER_STEP = 9   # deposit, xfwd, yfwd, kspace_z, yinv, xinv, gather, integrate, tick


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(spec, nd=2, nfg=2, maxb=2, charged=True):
    """Compulsory bytes per launch of each kernel: every input read once, every output
    written once (no re-reads, no atomics read-modify-write)."""
    N = spec.N
    nx, ny, nz = (int(v) for v in spec.grid)
    M = nx * ny * nz
    hs = nz * ny * (nx // 2 + 1) * 8          # one half-spectrum field, complex64
    npair = (nd + 1) // 2
    qb = 4 if charged else 0
    return {
        "deposit": N * (12 + 4 + qb) + npair * M * 8,
        "fft_x_fwd": npair * M * 8 + nd * hs,
        "fft_y_fwd": 2 * nd * hs,
        "kspace_z": nd * hs + 3 * nfg * hs,
        "fft_y_inv": 2 * 3 * nfg * hs,
        # the force records: paired planes, 12 bytes per point and force group
        "fft_x_inv": 3 * nfg * hs + nfg * M * 12,
        # x_t 12, flags 4, q, the grid force written 12, the records read once
        "gather": N * (12 + 4 + qb + 12) + nfg * M * 12,
        # x_t 12, x_{t-1} 12, x_{t+1} 12, noise r/w 24, flags 4, ids 4, the grid force 12,
        # bonds (row 4, partners 4*maxb, types 1*maxb), partner positions assumed cached
        "integrate": N * (12 + 12 + 12 + 24 + 4 + 4 + 12 + 4 + 5 * maxb),
    }


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def make_spec(scale):
    from tild_b200 import synth
    return synth.config_c2(scale=scale)


def cpu_sample(spec, threads, nsteps, warmup=1):
    """The reference's step on the host cores (oracle CpuStep, FP32).  Returns
    (particle-steps/s, seconds per step)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    nb, partner, btype = spec.partner_lists(2)
    sysm = oracle.System(Dim=3, L=spec.L, Nx=spec.grid, order=spec.order, x=spec.x, types=spec.types,
                         mass=np.ones(len(spec.species), np.float32),
                         mobility=np.ones(len(spec.species), np.float32), species=spec.species,
                         charges=spec.charges, nb=nb, partner=partner, btype=btype,
                         bond_k=np.array([spec.bond_k], np.float32), bond_req=np.array([0.0], np.float32),
                         bond_style=np.array([0], np.int32), potentials=spec.potentials, delt=spec.delt)
    cs = oracle.CpuStep(sysm, threads, seed=spec.seed)
    for _ in range(warmup):
        cs.step()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        cs.step()
    dt = time.perf_counter() - t0
    return spec.N * nsteps / dt, dt / nsteps


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(dist, x, device):
    """The largest x over all ranks, returned on every rank (x itself without a process
    group): whole-job times are the slowest rank's."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, ms):
    """Units processed by all ranks per second, every rank doing units_per_rank in the
    slowest rank's ms (replicas: the work per GPU is fixed as the GPU count grows)."""
    return world * units_per_rank / (ms * 1e-3)


def harness_path():
    return os.path.join(ROOT, "oracle", "_ref", "tild_ref_harness")


def reference_step_ms(spec, warmup, steps, workdir):
    """ms per step of the reference's own CUDA build (the unmodified MATILDA.FT sources built
    in place into oracle/_ref by oracle/ref_harness/Makefile) on `spec`: the harness reads
    the same data file and script as `matilda.ft -in`, sets the box up (finishInitialization),
    runs `warmup` doTimeStep calls, then times `steps` more with CUDA events.  Also returns
    the process wall time (set-up included)."""
    spec.log_freq = 1 << 30
    scr, _ = spec.write(workdir, steps=0)
    t0 = time.perf_counter()
    r = subprocess.run([harness_path(), os.path.basename(scr), "-", str(max(1, warmup)), str(steps)], cwd=workdir,
                       capture_output=True, text=True, timeout=3000)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError("reference harness rc=%d: %s" % (r.returncode, r.stderr[-500:]))
    ms = [float(ln.split()[1]) for ln in r.stdout.splitlines() if ln.startswith("ms_per_step")][0]
    return ms, wall


def reference_plain_jobs(jobs, time_steps, workdir):
    """Plain per-job form of the reference build on a job list [(spec, steps)]: one process
    per job, one after another, each job's time = its process wall time with the timed
    steps replaced by its own step count at the measured ms per step (set-up counted once,
    as a `matilda.ft -in job.in` run would)."""
    work, total, steady = 0.0, 0.0, 0.0
    for spec, steps in jobs:
        ms, wall = reference_step_ms(spec, 1, time_steps, workdir)
        total += wall - time_steps * ms * 1e-3 + steps * ms * 1e-3
        steady += steps * ms * 1e-3
        work += float(spec.N) * steps
    return {"value": work / total, "steady_state_value": work / steady, "unit": METRIC, "jobs": len(jobs),
            "particle_steps": work}


def every_kth(items, n):
    """n items spread evenly over the list (the whole list when n >= its length)."""
    if n >= len(items):
        return list(items)
    return [items[int(i * len(items) / n)] for i in range(n)]


def run_reference(args):
    """The reference arm: MATILDA.FT's own CUDA build (unmodified, through the harness) on
    this GPU, same workload and metric; rank 0 only.  Also times its plain per-job form on
    samples of the batched (C3) and served (C5) job lists that our arm runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import tempfile
    from tild_b200 import synth
    spec = make_spec(args.scale)
    base = {"impl": "reference", "metric": METRIC, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (numpy seed 2)", "config": bench_config(spec, args.gpus)}
    if not os.path.exists(harness_path()):
        return run_reference_port(args, base, "the reference build (oracle/_ref/tild_ref_harness) is absent")
    with tempfile.TemporaryDirectory() as d:
        ms, wall = reference_step_ms(spec, args.warmup, args.steps, d)
        value = spec.N / (ms * 1e-3)
        line = dict(base, value=value, ms_per_step=ms)
        line["cpu_baseline"] = {
            "value": value, "unit": METRIC, "cores": 1, "kind": "reference",
            "sample": "%d steps (after %d warm-up) of the full workload through MATILDA.FT's own CUDA build "
                      "(unmodified sources compiled for sm_100, PS_Box::doTimeStep driven by the harness, "
                      "CUDA events; one host thread drives it), on this B200; process wall %.1f s with set-up"
                      % (args.steps, args.warmup, wall)}
        line["e2e"] = {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        if not args.no_batch:
            c3 = [(s, args.c3_steps) for s in synth.config_c3(replicas=args.c3_replicas)]
            c3s = every_kth(c3, args.ref_jobs_c3)
            line["batched_reference"] = dict(
                reference_plain_jobs(c3s, args.ref_time_steps, d),
                workload="c3 plain per-job form of the reference build: %d of the %d replicas (every %gth), "
                         "%d steps each, one process per job" % (len(c3s), len(c3), len(c3) / len(c3s), args.c3_steps))
            c5 = c5_jobs(synth, args)
            c5s = every_kth(c5, args.ref_jobs_c5)
            line["served_reference"] = dict(
                reference_plain_jobs(c5s, args.ref_time_steps, d),
                workload="c5 plain per-job form of the reference build: %d of the %d jobs, one process per job "
                         "back to back" % (len(c5s), len(c5)))
    print(json.dumps(line), flush=True)
    return 0


def run_reference_port(args, base, why):
    """Fallback reference arm when the reference build is absent: the reference's
    algorithm restated on the host (oracle CpuStep, FP32, every host core) on a scaled
    replica of the workload sized to --ref-budget seconds."""
    threads = os.cpu_count() or 1
    probe = make_spec(args.scale / 64.0)
    _, t_probe = cpu_sample(probe, threads, 1, warmup=1)
    per_step_full = t_probe * 64.0
    s = min(1.0, args.ref_budget / max(1, args.steps + args.warmup) / per_step_full)
    s = max(s, 1.0 / 512.0)
    spec = make_spec(args.scale * s)
    value, sec = cpu_sample(spec, threads, args.steps, warmup=args.warmup)
    what = ("the full workload" if s >= 1.0 else
            "a replica of the workload scaled to %d particles, %s grid (same density and composition)"
            % (spec.N, "x".join(str(int(v)) for v in spec.grid)))
    line = dict(base, value=value, ms_per_step=sec * 1e3)
    line["cpu_baseline"] = {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                            "sample": "%d steps (after %d warm-up) of %s with the reference's algorithm restated "
                                      "on the host (stencil tables, deposit of every group, FP32 C2C FFTs); %s"
                                      % (args.steps, args.warmup, what, why)}
    line["e2e"] = {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    print(json.dumps(line), flush=True)
    return 0


def bench_config(spec, world):
    return {"workload": WORKLOAD, "particles": spec.N, "grid": [int(v) for v in spec.grid],
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (every kernel's operands exceed the 126 MB L2)"}


def c5_jobs(synth, args):
    """The served job list: BASELINE's size and length distribution (N log-uniform in
    [2e4, 1e6], 500-5,000 steps), --c5-jobs of them."""
    return synth.config_c5_jobs(njobs=args.c5_jobs, nmin=2.0e4, nmax=1.0e6, smin=500, smax=5000)


def cufft_times(torch, spec, nd, nfg, reps=20):
    """The spectral stage done with cuFFT (through torch.fft) and torch elementwise
    kernels, device-timed on the same grid and field counts:
      chain: what our five passes do -- R2C of the nd density fields, phi_f = u(k) rho_f,
             the three -i k_d phi_f, C2R of the 3*nfg gradient fields, float4 records;
      reference_form: the reference's own form (Box.cu:107-127, ps_potential.cu:41-125) --
             each field made complex, C2C forward, x 1/M, then per direction a complex
             multiply, a C2C inverse and the real part accumulated into the grid force;
      forward / inverse: the bare R2C and C2R transforms alone."""
    nx, ny, nz = (int(v) for v in spec.grid)
    dev = "cuda"
    L = [float(v) for v in spec.L]
    def kvec(n, l, half=False):
        k = torch.fft.rfftfreq(n, d=l / n, device=dev) if half else torch.fft.fftfreq(n, d=l / n, device=dev)
        return (2.0 * np.pi * k).to(torch.float32)
    kx, ky, kz = kvec(nx, L[0], True), kvec(ny, L[1]), kvec(nz, L[2])
    kxf = kvec(nx, L[0])
    rho = torch.rand((nd, nz, ny, nx), device=dev, dtype=torch.float32)
    uk = torch.rand((nfg, nz, ny, nx // 2 + 1), device=dev, dtype=torch.float32)
    ukf = torch.rand((nfg, nz, ny, nx), device=dev, dtype=torch.float32)
    spec_b = torch.randn((3 * nfg, nz, ny, nx // 2 + 1), device=dev, dtype=torch.complex64)
    M = nx * ny * nz

    def chain():
        rh = torch.fft.rfftn(rho, dim=(1, 2, 3))
        phi = uk * rh[:nfg]
        g = torch.stack([phi * (-1j * kx[None, None, None, :]), phi * (-1j * ky[None, None, :, None]),
                         phi * (-1j * kz[None, :, None, None])], 1).reshape(3 * nfg, nz, ny, nx // 2 + 1)
        r = torch.fft.irfftn(g, s=(nz, ny, nx), dim=(1, 2, 3)).reshape(nfg, 3, nz, ny, nx)
        return torch.cat([r.permute(0, 2, 3, 4, 1), torch.zeros((nfg, nz, ny, nx, 1), device=dev)], -1)

    def reference_form():
        gf = torch.zeros((nfg, 3, nz, ny, nx), device=dev, dtype=torch.float32)
        ks = (kxf[None, None, :], ky[None, :, None], kz[:, None, None])
        for f in range(nfg):
            c = rho[f].to(torch.complex64)
            F = torch.fft.fftn(c) * (1.0 / M)
            for d in range(3):
                gf[f, d] += torch.fft.ifftn(F * (-1j * ks[d] * ukf[f])).real
        return gf

    out = {}
    for name, fn in (("chain", chain), ("reference_form", reference_form),
                     ("forward", lambda: torch.fft.rfftn(rho, dim=(1, 2, 3))),
                     ("inverse", lambda: torch.fft.irfftn(spec_b, s=(nz, ny, nx), dim=(1, 2, 3)))):
        for _ in range(5):   # plans and the caching allocator settle first
            fn()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    del rho, uk, ukf, spec_b
    torch.cuda.empty_cache()
    return out


def job_box(tild_b200, spec):
    return tild_b200.box_from_spec(spec, options={"write_files": 0})


def pct(v, q):
    return float(np.percentile(np.asarray(v, np.float64), q)) if len(v) else None


def run_batched(tild_b200, synth, args):
    """C3: uneven diblock replicas stepped as one batch (tild_batch_*: every stage of a
    step is one kernel launch over all replicas, a step is one CUDA graph), against the same
    jobs run one after another (plain per-job form) and in the job pool (each replica its
    own graph on its own stream).  Wall clock from the first endBox (or submit) to the last
    result on the host; boxes are built on the host before the clock starts in every form."""
    specs = synth.config_c3(replicas=args.c3_replicas)
    steps = args.c3_steps
    work = float(sum(s.N for s in specs)) * steps
    boxes = [job_box(tild_b200, s) for s in specs]
    t0 = time.perf_counter()
    for b in boxes:
        b.command("endBox")
        b.step(steps)
        b.positions()
        b.close()
    plain_s = time.perf_counter() - t0
    boxes = [job_box(tild_b200, s) for s in specs]
    t0 = time.perf_counter()
    for b in boxes:
        b.command("endBox")
    with tild_b200.Batch() as batch:
        for b in boxes:
            batch.add(b)
        batch.step(steps)
    for b in boxes:
        b.positions()
    batch_s = time.perf_counter() - t0
    for b in boxes:
        b.close()
    boxes = [job_box(tild_b200, s) for s in specs]
    with tild_b200.Pool(mem_budget_bytes=args.pool_budget_gb << 30) as pool:
        t0 = time.perf_counter()
        ids = [pool.submit(b, steps) for b in boxes]
        for jid, s in zip(ids, specs):
            pool.wait(jid)
            pool.result(jid, s.N)
        pool_s = time.perf_counter() - t0
    for b in boxes:
        b.close()
    return {"workload": "c3: %d diblock replicas, %d steps each, N %d..%d (total %d), grids %d^3..%d^3"
                        % (len(specs), steps, min(s.N for s in specs), max(s.N for s in specs),
                           sum(s.N for s in specs), min(int(s.grid[0]) for s in specs),
                           max(int(s.grid[0]) for s in specs)),
            "value": work / batch_s, "unit": METRIC, "plain_value": work / plain_s,
            "pool_value": work / pool_s, "speedup_vs_plain": plain_s / batch_s, "batched_s": batch_s,
            "plain_s": plain_s, "pool_s": pool_s,
            "form": "tild_batch: one kernel launch per step stage over all replicas (10 per step, one CUDA "
                    "graph); re-sorts every 10 steps as branches of one graph",
            "timing": "wall clock, host, includes allocation, upload, first sort, graph capture and result copies"}


def pool_capacity(tild_b200, args, jobs):
    """Throughput of the pool on a job mix submitted all at once (particle-steps/s, wall
    clock from the first submit to the last result)."""
    boxes = [job_box(tild_b200, s) for s, _ in jobs]
    with tild_b200.Pool(mem_budget_bytes=args.pool_budget_gb << 30) as pool:
        t0 = time.perf_counter()
        ids = [pool.submit(b, n) for b, (_, n) in zip(boxes, jobs)]
        for jid, (s, _) in zip(ids, jobs):
            pool.wait(jid)
            pool.result(jid, s.N)
        dt = time.perf_counter() - t0
    for b in boxes:
        b.close()
    return float(sum(s.N * n for s, n in jobs)) / dt


def run_served(tild_b200, synth, args):
    """C5: jobs arriving as a Poisson process at an offered load of `c5_load` times the
    pool's throughput on the same job mix (measured first, all jobs submitted at once),
    admitted by the pool as memory frees up; latency = completion - arrival.  The same
    jobs run alone give the plain per-job service times."""
    jobs = c5_jobs(synth, args)
    work = np.array([s.N * n for s, n in jobs], np.float64)
    capacity = pool_capacity(tild_b200, args, jobs)
    boxes = [job_box(tild_b200, s) for s, _ in jobs]
    service = []
    for b, (s, n) in zip(boxes, jobs):
        t0 = time.perf_counter()
        b.command("endBox")
        b.step(n)
        b.positions()
        b.thermo_raw()
        service.append(time.perf_counter() - t0)
        b.close()
    rate = args.c5_load * capacity / float(work.mean())   # jobs per second
    arrivals = np.cumsum(np.random.default_rng(5).exponential(1.0 / rate, len(jobs)))
    boxes = [job_box(tild_b200, s) for s, _ in jobs]
    lat, spans = [], []
    with tild_b200.Pool(mem_budget_bytes=args.pool_budget_gb << 30) as pool:
        t0 = time.perf_counter()
        ids = []
        for b, a in zip(boxes, arrivals):
            dt = t0 + a - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            ids.append(pool.submit(b, jobs[len(ids)][1]))
        for jid, (s, _) in zip(ids, jobs):
            pool.wait(jid)
            pool.result(jid, s.N)
            st = pool.status(jid)
            lat.append(st["done_s"] - st["submit_s"])
            spans.append((st["submit_s"], st["done_s"]))
    for b in boxes:
        b.close()
    makespan = max(d for _, d in spans) - min(a for a, _ in spans)
    return {"workload": "c5: %d jobs (diblock or coacervate), N %d..%d, %d..%d steps, Poisson arrivals at %.0f%% of "
                        "the pool's throughput on this mix (%.1f jobs/s)" % (len(jobs), min(s.N for s, _ in jobs),
                                                                             max(s.N for s, _ in jobs),
                                                                             min(n for _, n in jobs),
                                                                             max(n for _, n in jobs),
                                                                             100 * args.c5_load, rate),
            "capacity": capacity,
            "value": float(work.sum()) / makespan, "unit": METRIC, "latency_p50_s": pct(lat, 50),
            "latency_p99_s": pct(lat, 99), "plain_value": float(work.sum()) / sum(service),
            "plain_service_p50_s": pct(service, 50), "plain_service_p99_s": pct(service, 99),
            "timing": "wall clock; latency from submit to result available; plain = each job alone, back to back"}


def run_ours(args):
    import torch
    import tild_b200
    world, rank, local, dist = dist_setup(args)
    torch.cuda.set_device(local)
    spec = make_spec(args.scale)
    stream = torch.cuda.Stream(device=local)
    opts = {"write_files": 0, "autotune": 0 if args.no_autotune else 1}
    opts.update(json.loads(args.box_options))
    box = tild_b200.box_from_spec(spec, device=local, options=opts)
    box.set_stream(stream.cuda_stream)
    box.command("endBox")
    info = box.info()
    tiles = box.describe()["tiles"]
    for _ in range(args.warmup):
        box.step(1)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        box.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(dist, e0.elapsed_time(e1), "cuda")
    if dist:
        dist.barrier()
    value = whole_job_rate(world, spec.N * args.steps, ms)

    # end to end through the C ABI: pinned host positions -> S steps -> host positions
    S = args.e2e_steps
    hx = torch.empty((spec.N, 3), dtype=torch.float32).pin_memory()
    hx.copy_(torch.from_numpy(box.positions()))
    hout = torch.empty_like(hx).pin_memory()
    import ctypes
    L = tild_b200.lib()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    tild_b200._check(L.tild_box_set_positions(box._h, ctypes.c_void_p(hx.data_ptr())))
    tild_b200._check(L.tild_box_step(box._h, S))
    tild_b200._check(L.tild_box_get_positions(box._h, ctypes.c_void_p(hout.data_ptr())))
    f1.record(stream)
    torch.cuda.synchronize()
    ems = max_over_ranks(dist, f0.elapsed_time(f1), "cuda")
    e2e = whole_job_rate(world, spec.N * S, ems)

    # per-kernel durations: instrumented launches (an event after every kernel)
    box.set_option("stage_timing", 1)
    box.step(args.profile_steps)
    box.set_option("stage_timing", 0)
    st = np.zeros(8)
    n = ctypes.c_int()
    L.tild_box_stage_times(box._h, st.ctypes.data_as(ctypes.c_void_p), 8, ctypes.byref(n))
    stage_s = dict(zip(STAGES, st[: n.value]))
    ab = algorithmic_bytes(spec, nd=info.n_density_fields, nfg=info.n_force_groups, charged=True)
    dom = max(stage_s, key=lambda k: stage_s[k])
    peak, peak_kind = peaks()
    achieved = ab[dom] / stage_s[dom] / 1e9
    traffic = None
    tf = os.path.join(ROOT, "profiles", "dram_traffic_c2.json")
    if args.scale == 1.0 and os.path.exists(tf):   # captured on the full-size workload only
        traffic = json.load(open(tf)).get(KERNEL_NAMES[dom])
    step_bytes = sum(ab.values())
    cf = cufft_times(torch, spec, info.n_density_fields, info.n_force_groups)
    ours_fft = sum(stage_s[k] for k in ("fft_x_fwd", "fft_y_fwd", "kspace_z", "fft_y_inv", "fft_x_inv")) * 1e3
    fft_cmp = {"ours_ms": ours_fft, "cufft_chain_ms": cf["chain"], "reference_form_ms": cf["reference_form"],
               "cufft_r2c_c2r_only_ms": cf["forward"] + cf["inverse"],
               "note": "ours = our x/y/z passes (R2C, k-space combine, -ik gradients, C2R, float4 force records); "
                       "cufft_chain = the same work as cuFFT R2C/C2R plus torch elementwise kernels; "
                       "reference_form = the reference's C2C forward, 1/M, and per direction multiply, C2C "
                       "inverse and real part, with cuFFT; cufft_r2c_c2r_only = the bare transforms"}
    # sorts inside the timed region: every sort_interval steps, 10 kernels each (keys, a
    # three-kernel scan, new slots, permute, and for the CSR bond rows a second scan and
    # their permute)
    si = 10
    nsort = (args.warmup + args.steps) // si - args.warmup // si

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            threads = os.cpu_count() or 1
            cv, csec = cpu_sample(spec, threads, args.cpu_steps, warmup=0)
            cpu = {"value": cv, "unit": METRIC, "cores": threads, "kind": "port",
                   "sample": "%d full step(s) of the same workload, reference algorithm restated on the host "
                             "(oracle CpuStep, FP32, OpenMP + scipy.fft), %.1f s per step" % (args.cpu_steps, csec)}
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (numpy seed 2)",
            "config": bench_config(spec, world),
            "rng": "philox",
            "tiles": {"bricks_per_cta": tiles["codes"], "threads": tiles["threads"], "gather": tiles["gather"],
                      "deposit_bricks_per_cta": tiles["deposit_codes"], "deposit_threads": tiles["deposit_threads"],
                      "autotuned": not args.no_autotune},
            "step_algorithmic_gb": step_bytes / 1e9,
            "roofline": {"bound": "hbm", "kernel": KERNEL_NAMES[dom], "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes": ab[dom],
                         "kernel_ms": {k: v * 1e3 for k, v in stage_s.items()},
                         # every kernel of the step: algorithmic bytes / CUDA-event time, of peak
                         "kernels": {KERNEL_NAMES[k]: {"ms": v * 1e3, "algorithmic_mb": ab[k] / 1e6,
                                                       "gbs": ab[k] / v / 1e9, "frac": ab[k] / v / 1e9 / peak}
                                     for k, v in stage_s.items() if v > 0},
                         "step_algorithmic_gbs": step_bytes / (ms / args.steps * 1e-3) / 1e9,
                         "step_frac": step_bytes / (ms / args.steps * 1e-3) / 1e9 / peak},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": METRIC, "steps_per_job": S,
                    "h2d_bytes_per_step": spec.N * 12 / S, "d2h_bytes_per_step": spec.N * 12 / S},
            "fft_vs_cufft": fft_cmp,
            "gpu_launches": KERNELS_PER_STEP * args.steps + 10 * nsort,
            "clocks": clk.summary(),
        }
    box.close()
    if rank == 0:
        if world == 1 and not args.no_batch:
            from tild_b200 import synth
            line["batched"] = run_batched(tild_b200, synth, args)
            line["served"] = run_served(tild_b200, synth, args)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="workload scale (tests only)")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched (C3) and served (C5) runs")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the density rule's tiles (profiling: fewer launches before the steps)")
    ap.add_argument("--box-options", default="{}",
                    help="JSON of box options, e.g. fixed tiles for profiling: "
                         '\'{"tile_codes": 4, "deposit_codes": 8, "deposit_threads": 128}\'')
    ap.add_argument("--c3-replicas", type=int, default=64)
    ap.add_argument("--c3-steps", type=int, default=2000)
    ap.add_argument("--c5-jobs", type=int, default=24, help="served jobs (the stated stream has 2,000)")
    ap.add_argument("--c5-load", type=float, default=0.8)
    ap.add_argument("--pool-budget-gb", type=int, default=150)
    ap.add_argument("--ref-budget", type=float, default=150.0, help="seconds for the host-port fallback arm")
    ap.add_argument("--ref-jobs-c3", type=int, default=16, help="C3 replicas the reference arm times")
    ap.add_argument("--ref-jobs-c5", type=int, default=8, help="C5 jobs the reference arm times")
    ap.add_argument("--ref-time-steps", type=int, default=30, help="timed steps per reference job")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    return run_reference(args) if args.impl == "reference" else run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
