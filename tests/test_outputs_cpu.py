"""CPU tests of the run-time outputs' host side: the output words (trajFreq, trajFileName,
fieldFreq [logspace s], gsdFreq [logspace s], gsdName; PS_Box_initialization.cu:171-215,
310-316), and the files endBox writes before any device work -- the GSD trajectory's first
frame (GSDinit + writeGSDtraj, PS_Box_gsdUtils.cu:14-168, 586-608) and the headers of the
group density files (Box::initBinaryDataFile, Box.cu:552-570).  The GSD file is read with
the test reader (oracle/gsd_reader.py) and, where it has been built, with the reference's
own gsd.c reader (oracle/_ref/gsd_dump); both must agree byte for byte."""
import os
import subprocess

import numpy as np
import pytest

import gsd_reader
import tild_b200
from tild_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GSD_DUMP = os.path.join(ROOT, "oracle", "_ref", "gsd_dump")
ANGLES = [dict(style="harmonic", k=3.0, theta=120.0)]


def spec():
    return synth.small_system(seed=21, charges=True, angle_params=ANGLES)


def end_box(b):
    """endBox: the host set-up (and the files it writes) runs first; without a GPU the
    device set-up then fails with TILD_ERR_CUDA, which is expected here."""
    try:
        b.command("endBox")
    except tild_b200.TildError as e:
        assert e.code == 4, str(e)


def box_with_files(s, tmp_path, extra=()):
    b = tild_b200.box_from_spec(s, options={"write_files": 1}, base_dir=str(tmp_path))
    b.command("group grpB types B")
    for line in extra:
        b.command(line)
    return b


def test_output_words_parse():
    b = tild_b200.Box(0)
    for line in ["Dim 3", "trajFreq 25", "trajFileName run.lammpstrj", "fieldFreq 10 logspace 1.5",
                 "gsd_freq 4 log_space 2.0", "gsdName run.gsd"]:
        b.command(line)
    d = b.describe()
    assert d["trajFreq"] == 25 and d["trajFileName"] == "run.lammpstrj"
    assert d["fieldFreq"] == 10 and abs(d["logScaleFields"] - 1.5) < 1e-7
    assert d["gsdFreq"] == 4 and abs(d["logScaleGSD"] - 2.0) < 1e-7 and d["gsdName"] == "run.gsd"
    b.close()
    b = tild_b200.Box(0)
    b.command("Dim 3")
    for bad in ["fieldFreq 5 every 2", "gsdFreq 5 linear 2"]:
        with pytest.raises(tild_b200.TildError) as e:
            b.command(bad)
        assert e.value.code == 2 and "invalid option" in str(e.value)
    b.close()


def test_density_file_headers(tmp_path):
    s = spec()
    b = box_with_files(s, tmp_path)
    end_box(b)
    b.close()
    names = ["grpB", "all", "A", "B", "charges"]
    for nm in names:
        raw = open(os.path.join(tmp_path, "density-%s.bin" % nm), "rb").read()
        head = np.frombuffer(raw[:16], np.int32)
        assert head[0] == 3 and list(head[1:]) == [int(v) for v in s.grid]
        assert np.array_equal(np.frombuffer(raw[16:28], np.float32), np.asarray(s.L, np.float32))
        # frames (M floats each) follow the header; a GPU run may have added some
        assert (len(raw) - 28) % (4 * int(np.prod(s.grid))) == 0


def expected_first_frame(s):
    N = s.N
    x = np.asarray(s.x, np.float32)
    Lh = (np.float32(0.5) * np.asarray(s.L, np.float32)).astype(np.float32)
    pairs = []
    part = [[] for _ in range(N)]
    for i, j in np.asarray(s.bonds):
        part[i].append(j)
        part[j].append(i)
    for p in range(N):           # each bond from its lower end, in bondedTo order
        for q in part[p]:
            if q > p:
                pairs.append((p, q))
    ang = np.asarray(s.angles, np.uint32).reshape(-1, 3).copy()   # in input order, ends i1 < i3
    swap = ang[:, 2] < ang[:, 0]
    ang[swap, 0], ang[swap, 2] = ang[swap, 2], ang[swap, 0].copy()
    types = np.zeros((len(s.species) + 1, 10), np.int8)
    for t in range(len(s.species) + 1):
        nm = ("type%d" % t).encode()
        types[t, :len(nm)] = np.frombuffer(nm, np.int8)
    return {
        "configuration/step": np.array([0], np.uint64),
        "configuration/dimensions": np.array([3], np.uint8),
        "configuration/box": np.array(list(s.L) + [0, 0, 0], np.float32),
        "particles/N": np.array([N], np.uint32),
        "particles/mass": np.asarray(s.masses, np.float32)[s.types],
        "particles/typeid": (np.asarray(s.types) + 1).astype(np.uint32),
        "log/particles/moleculeid": (np.asarray(s.mol) + 1).astype(np.uint32),
        "particles/types": types,
        "bonds/N": np.array([len(pairs)], np.uint32),
        "bonds/typeid": np.zeros(len(pairs), np.uint32),
        "bonds/group": np.array(pairs, np.uint32).reshape(-1, 2),
        "angles/N": np.array([len(s.angles)], np.uint32),
        "angles/typeid": np.asarray(s.angle_types, np.uint32),
        "angles/group": ang,
        "particles/position": (x - Lh).astype(np.float32),
        "particles/charge": np.asarray(s.charges, np.float32),
    }


def test_gsd_first_frame_written_at_endbox(tmp_path):
    s = spec()
    b = box_with_files(s, tmp_path, ["gsdName first.gsd"])
    end_box(b)
    b.close()
    g = gsd_reader.GsdFile(os.path.join(tmp_path, "first.gsd"))
    assert g.application == "gpu-tild" and g.schema == "hoomd"
    assert g.schema_version == gsd_reader.version(1, 4) and g.gsd_version == gsd_reader.version(2, 0)
    exp = expected_first_frame(s)
    assert [c[0] for c in g.chunk_order(0)] == list(exp)   # names in the reference's write order
    fr = g.frame(0)
    for k, v in exp.items():
        assert fr[k].dtype == v.dtype and fr[k].shape == v.shape, k
        assert np.array_equal(fr[k], v), k


def dump_reference_reader(path):
    r = subprocess.run([GSD_DUMP, path], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.splitlines()
    nframes = int(lines[0].split()[1])
    chunks = {}
    for ln in lines[5:]:
        f, name, N, M, typ, hexdata = (ln.split(" ") + [""])[:6]
        chunks[(int(f), name)] = (int(N), int(M), int(typ), bytes.fromhex(hexdata))
    return nframes, chunks


def compare_with_reference_reader(path):
    g = gsd_reader.GsdFile(path)
    nframes, chunks = dump_reference_reader(path)
    assert nframes == g.nframes
    mine = {}
    for f in range(g.nframes):
        for (name, N, M, typ) in g.chunk_order(f):
            a = g.frame(f)[name]
            mine[(f, name)] = (N, M, typ, a.tobytes())
    assert mine == chunks


@pytest.mark.skipif(not os.path.exists(GSD_DUMP), reason="reference GSD reader not built (needs the reference sources)")
def test_gsd_file_reads_identically_with_the_reference_reader(tmp_path):
    s = spec()
    b = box_with_files(s, tmp_path)
    end_box(b)
    b.close()
    compare_with_reference_reader(os.path.join(tmp_path, "traj.gsd"))


def test_gsd_reader_rejects_corrupt_files(tmp_path):
    s = spec()
    b = box_with_files(s, tmp_path)
    end_box(b)
    b.close()
    raw = bytearray(open(os.path.join(tmp_path, "traj.gsd"), "rb").read())
    bad = bytearray(raw)
    bad[0] ^= 0xFF                                   # magic
    (tmp_path / "bad1.gsd").write_bytes(bytes(bad))
    with pytest.raises(ValueError, match="magic"):
        gsd_reader.GsdFile(str(tmp_path / "bad1.gsd"))
    (tmp_path / "bad2.gsd").write_bytes(bytes(raw[:2000]))   # cut inside the data
    with pytest.raises(ValueError):
        gsd_reader.GsdFile(str(tmp_path / "bad2.gsd"))


def test_reader_on_the_reference_trajectory(tmp_path):
    """The GSD file the reference itself wrote (outputs_ref.npz, make_ref_outputs.py): the
    test reader finds its frames and chunks, identically to the reference's reader."""
    z = np.load(os.path.join(ROOT, "tests", "golden", "outputs_ref.npz"))
    path = str(tmp_path / "ref.gsd")
    (tmp_path / "ref.gsd").write_bytes(z["gsd"].tobytes())
    g = gsd_reader.GsdFile(path)
    assert g.nframes == 4 and g.application == "gpu-tild"
    assert [c[0] for c in g.chunk_order(1)] == ["configuration/step", "particles/position", "particles/charge"]
    assert [int(g.frame(f)["configuration/step"][0]) & 0xFFFFFFFF for f in range(4)] == [0, 5, 10, 12]
    if os.path.exists(GSD_DUMP):
        compare_with_reference_reader(path)


def test_2d_box_outputs_at_endbox(tmp_path):
    """A 2-D box: density headers carry Dim 2 with two grid sizes and lengths, and the GSD
    frame has the reference's 2-D box (Lz = 5.0) and particles on the plane z = 0 - L/2
    only through x and y (z written as 0)."""
    s = synth.small_system(seed=24, dim=2, grid=(16, 18, 1), charges=True)
    b = tild_b200.box_from_spec(s, options={"write_files": 1}, base_dir=str(tmp_path))
    end_box(b)
    b.close()
    raw = open(os.path.join(tmp_path, "density-all.bin"), "rb").read()
    assert np.frombuffer(raw[:4], np.int32)[0] == 2
    assert list(np.frombuffer(raw[4:12], np.int32)) == [16, 18]
    assert np.array_equal(np.frombuffer(raw[12:20], np.float32), np.asarray(s.L[:2], np.float32))
    assert (len(raw) - 20) % (4 * 16 * 18) == 0
    fr = gsd_reader.GsdFile(os.path.join(tmp_path, "traj.gsd")).frame(0)
    assert np.array_equal(fr["configuration/box"], np.array([s.L[0], s.L[1], 5.0, 0, 0, 0], np.float32))
    x = np.asarray(s.x, np.float32)
    Lh = np.float32(0.5) * np.asarray(s.L[:2], np.float32)
    pos = fr["particles/position"]
    assert np.array_equal(pos[:, :2], (x - Lh).astype(np.float32)) and not pos[:, 2].any()
