"""Run-time outputs on the GPU (PS_Box.cu:166-234): lammpstrj frames, group density
frames (density-<group>.bin) and the GSD trajectory, written from asynchronous device
snapshots during NVT.

Checks:
  * schedule: the frame steps follow trajFreq / fieldFreq (with logspace growth) /
    gsdFreq exactly as doTimeStep does, plus the closing frames of NVT;
  * content, against an identical deterministic box stepped without outputs: lammpstrj
    text identical to the reference's format applied to those positions (one wrap, %f);
    GSD positions = x - L/2 bit for bit; density frames within the density tolerance of
    the parity tests (|drho| <= 1e-6 max|rho|) of the FP64 oracle at the positions each
    frame's step started from;
  * the GSD file reads identically with the reference's own reader when it is built;
  * against the reference's own outputs for the same script (tests/golden/outputs_ref.npz,
    written by the reference build through make_ref_outputs.py), with cuRAND-compatible
    noise: frame steps, headers, ids, types and topology exactly; positions within 1e-3
    (12 steps of trajectories that differ only by float summation order); densities within
    2e-3 max|rho|.  The reference's GSD bond and angle totals count data-file bonds and
    angles twice and pad the lists with zero rows; that defect is checked, not copied.
"""
import os

import numpy as np
import pytest

import gsd_reader
import oracle
import tild_b200
from conftest import spec_to_system
from test_outputs_cpu import GSD_DUMP, compare_with_reference_reader
from tild_b200 import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "outputs_ref.npz")


def spec():
    return synth.small_system(seed=23, order=3, charges=True,
                              angle_params=[dict(style="harmonic", k=3.0, theta=120.0)])


def run_with_outputs(s, tmp_path, words, nsteps):
    b = tild_b200.box_from_spec(s, options={"write_files": 1, "deterministic": 1}, base_dir=str(tmp_path))
    for w in words:
        b.command(w)
    b.command("endBox")
    b.run_nvt(nsteps)
    x = b.positions()
    b.close()
    return x


def positions_by_step(s, nsteps):
    """xs[k] = positions after k steps of an identical box that writes nothing."""
    xs = []
    with tild_b200.box_from_spec(s, options={"write_files": 0, "deterministic": 1}) as b:
        b.command("endBox")
        xs.append(b.positions())
        for _ in range(nsteps):
            b.step(1)
            xs.append(b.positions())
    return xs


def field_schedule(freq, scale, nsteps):
    steps = []
    for i in range(nsteps):
        if freq > 0 and i % freq == 0:
            steps.append(i)
            if i > 1 and scale:
                freq = int(np.float32(freq) * np.float32(scale))
    return steps


def read_bin(path):
    raw = open(path, "rb").read()
    dim = int(np.frombuffer(raw[:4], np.int32)[0])
    nx = np.frombuffer(raw[4:4 + 4 * dim], np.int32)
    L = np.frombuffer(raw[4 + 4 * dim:4 + 8 * dim], np.float32)
    M = int(np.prod(nx))
    body = np.frombuffer(raw[4 + 8 * dim:], np.float32)
    assert body.size % M == 0
    return dim, nx, L, body.reshape(-1, M)


def lammpstrj_text(step, x, s):
    """PS_Box::writeLammpsTraj (PS_Box.cu:750-795) applied to positions x (float32, N x Dim):
    one wrap per coordinate, "%f " per dimension, then "%f" of 0 for a missing z."""
    D = s.dim
    L = np.asarray(s.L, np.float32)
    out = ["ITEM: TIMESTEP\n%d\nITEM: NUMBER OF ATOMS\n%d\n" % (step, s.N), "ITEM: BOX BOUNDS pp pp pp\n",
           "%f %f\n%f %f\n%f %f\n" % (0.0, L[0], 0.0, L[1], 0.0, L[2] if D == 3 else 1.0),
           "ITEM: ATOMS id type mol x y z\n"]
    for p in range(s.N):
        row = "%d %d %d  " % (p + 1, s.types[p] + 1, s.mol[p] + 1)
        for j in range(D):
            v = np.float32(x[p, j])
            if v > L[j]:
                v = np.float32(v - L[j])
            elif v < np.float32(0.0):
                v = np.float32(v + L[j])
            row += "%f " % v
        row += "%f" % 0.0 * (3 - D)
        out.append(row + "\n")
    return "".join(out)


def test_density_frames_schedule_and_content(tmp_path):
    s = spec()
    n = 12
    xfin = run_with_outputs(s, tmp_path, ["fieldFreq 2 logspace 2.0", "group grpA types A"], n)
    xs = positions_by_step(s, n)
    assert np.array_equal(xfin, xs[n])              # the outputs did not disturb the run
    sched = field_schedule(2, 2.0, n)
    assert sched == [0, 2, 4, 8]
    sysm = spec_to_system(s)
    sysm.user_groups = [("grpA", ["A"])]
    for name, _, _ in oracle.groups(sysm):
        dim, nx, L, frames = read_bin(os.path.join(tmp_path, "density-%s.bin" % name))
        assert dim == 3 and list(nx) == list(s.grid) and np.array_equal(L, np.asarray(s.L, np.float32))
        # one frame per scheduled step, then the closing frame: the densities the last step
        # started from (writeFields after the loop reuses the groups' d_rho)
        assert frames.shape[0] == len(sched) + 1, name
        for f, step in enumerate(sched + [n - 1]):
            dens, _, _ = oracle.densities(sysm, x=xs[step].astype(np.float32))
            ref = dens[name][0]
            assert np.abs(frames[f] - ref).max() <= 1e-6 * np.abs(ref).max(), (name, step)


def test_lammpstrj_frames_match_reference_format(tmp_path):
    s = spec()
    n = 10
    run_with_outputs(s, tmp_path, ["trajFreq 3", "trajFileName run.lammpstrj"], n)
    xs = positions_by_step(s, n)
    expect = "".join(lammpstrj_text(i, xs[i + 1], s) for i in range(n) if i % 3 == 0)
    got = open(os.path.join(tmp_path, "run.lammpstrj")).read()
    assert got == expect


def test_lammpstrj_frames_of_a_2d_box(tmp_path):
    s = synth.small_system(seed=25, order=3, dim=2, grid=(16, 18, 1), charges=True)
    n = 4
    run_with_outputs(s, tmp_path, ["trajFreq 2"], n)
    xs = positions_by_step(s, n)
    expect = "".join(lammpstrj_text(i, xs[i + 1], s) for i in range(n) if i % 2 == 0)
    assert open(os.path.join(tmp_path, "traj.lammpstrj")).read() == expect


def test_gsd_frames(tmp_path):
    s = spec()
    n = 7
    run_with_outputs(s, tmp_path, ["gsdFreq 2"], n)
    xs = positions_by_step(s, n)
    g = gsd_reader.GsdFile(os.path.join(tmp_path, "traj.gsd"))
    # the set-up frame is replaced at step 0 (the file is created again while the box's step
    # count is 0); then steps 2, 4, 6 and the end of the run (step count 7)
    steps = [0, 2, 4, 6, 7]
    assert g.nframes == len(steps)
    Lh = np.float32(0.5) * np.asarray(s.L, np.float32)
    for f, st in enumerate(steps):
        fr = g.frame(f)
        assert fr["configuration/step"][0] == st
        x = xs[min(st + 1, n)]
        assert np.array_equal(fr["particles/position"], (x - Lh).astype(np.float32)), st
        assert np.array_equal(fr["particles/charge"], np.asarray(s.charges, np.float32))
        names = [c[0] for c in g.chunk_order(f)]
        if f == 0:
            assert len(names) == 16 and names[0] == "configuration/step"
        else:
            assert names == ["configuration/step", "particles/position", "particles/charge"]


def test_gsd_index_grows_past_its_first_region(tmp_path):
    """61 frames of 3 chunks outgrow the 128-entry index written at creation; the file
    stays readable by both readers."""
    s = spec()
    n = 60
    run_with_outputs(s, tmp_path, ["gsdFreq 1"], n)
    path = os.path.join(tmp_path, "traj.gsd")
    g = gsd_reader.GsdFile(path)
    assert g.nframes == n + 1 and g.index_allocated > 128
    assert [int(g.frame(f)["configuration/step"][0]) for f in range(g.nframes)] == list(range(n)) + [n]
    if os.path.exists(GSD_DUMP):
        compare_with_reference_reader(path)


# ---- against the reference's own outputs --------------------------------------------

def _ref():
    if not os.path.exists(GOLDEN):
        pytest.skip("outputs_ref.npz not generated")
    return np.load(GOLDEN)


def _run_reference_script(z, tmp_path):
    (tmp_path / "outputs.data").write_text(str(z["data"]))
    b = tild_b200.Box(0, base_dir=str(tmp_path), options={"write_files": 1, "rng": 1})
    for line in str(z["script"]).splitlines():
        if not line.strip() or line.startswith("box") or line.startswith("run"):
            continue
        b.command(line)
    b.run_nvt(int(z["nsteps"]))
    b.close()


def _periodic(d, L):
    d = np.abs(d)
    return np.minimum(d, L - d)


def _parse_traj(text):
    lines = text.splitlines()
    frames, k = [], 0
    while k < len(lines):
        assert lines[k] == "ITEM: TIMESTEP"
        step, n = int(lines[k + 1]), int(lines[k + 3])
        head = lines[k + 4:k + 9]
        rows = [ln.split() for ln in lines[k + 9:k + 9 + n]]
        frames.append((step, head, np.array([r[:3] for r in rows], int), np.array([r[3:] for r in rows], float)))
        k += 9 + n
    return frames


def test_outputs_match_reference_files(tmp_path):
    z = _ref()
    _run_reference_script(z, tmp_path)
    L = None
    # lammpstrj
    ref, got = _parse_traj(str(z["traj"])), _parse_traj(open(os.path.join(tmp_path, "traj.lammpstrj")).read())
    assert [f[0] for f in got] == [f[0] for f in ref]
    for (s1, h1, i1, x1), (s2, h2, i2, x2) in zip(got, ref):
        assert h1 == h2 and np.array_equal(i1, i2)
        L = np.array([float(v.split()[1]) for v in h2[1:4]])
        assert _periodic(x1 - x2, L).max() <= 1e-3
    # density frames
    for key in z.files:
        if not key.startswith("density_"):
            continue
        name = key[len("density_"):]
        path = os.path.join(tmp_path, "density-%s.bin" % name)
        mine, theirs = open(path, "rb").read(), z[key].tobytes()
        hdr = 4 + 8 * 3
        assert mine[:hdr] == theirs[:hdr] and len(mine) == len(theirs), name
        a = np.frombuffer(mine[hdr:], np.float32)
        r = np.frombuffer(theirs[hdr:], np.float32)
        assert np.abs(a - r).max() <= 2e-3 * np.abs(r).max(), name
    # GSD: same frames, chunk lists, topology; positions within the trajectory tolerance
    (tmp_path / "ref.gsd").write_bytes(z["gsd"].tobytes())
    gr, gm = gsd_reader.GsdFile(str(tmp_path / "ref.gsd")), gsd_reader.GsdFile(os.path.join(tmp_path, "traj.gsd"))
    assert gm.nframes == gr.nframes
    assert (gm.application, gm.schema, gm.schema_version) == (gr.application, gr.schema, gr.schema_version)
    topo = ("bonds/", "angles/")
    for f in range(gr.nframes):
        om, orf = gm.chunk_order(f), gr.chunk_order(f)
        assert [(c[0], c[2], c[3]) for c in om] == [(c[0], c[2], c[3]) for c in orf]
        fm, fr = gm.frame(f), gr.frame(f)
        for name in fr:
            if name == "configuration/step":   # the reference fills only the low 32 bits
                assert int(fm[name][0]) == int(fr[name][0]) & 0xFFFFFFFF
            elif name == "particles/position":
                assert _periodic(fm[name] - fr[name], L).max() <= 1e-3
            elif name in ("bonds/N", "angles/N"):
                # the reference counts data-file bonds and angles twice
                assert int(fr[name][0]) == 2 * int(fm[name][0]) > 0, name
            elif name.startswith(topo):
                n = fm[name].shape[0]
                assert np.array_equal(fm[name], fr[name][:n]) and not fr[name][n:].any(), name
            else:
                assert fm[name].shape == fr[name].shape and np.array_equal(fm[name], fr[name]), (f, name)
    # thermo log rows: same steps, energies within 1e-4 relative
    rows = lambda t: [list(map(float, ln.split())) for ln in t.splitlines() if ln.strip()]
    rm, rr = rows(open(os.path.join(tmp_path, "ps_data.dat")).read()), rows(str(z["ps_data"]))
    assert [r[0] for r in rm] == [r[0] for r in rr]
    for a, b in zip(rm, rr):
        assert np.allclose(a[1:], b[1:], rtol=1e-4, atol=1e-6)
