"""CPU tests of the C ABI and host logic: the library loads, exports every symbol the
header declares, and the script/data-file front end (PS_Box::readInput,
readDataConfig) parses and rejects inputs like the reference -- no GPU call made."""
import os
import re

import numpy as np
import pytest

import tild_b200
from tild_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "tild_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tild_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = tild_b200.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(tild_b200._SIGS), "binding signatures must cover the header"


def test_version_string():
    assert b"sm_100a" in tild_b200.lib().tild_version()


def test_parse_script_words_like_read_input():
    b = tild_b200.Box(0)
    for line in ["# comment", "", "Dim 3 grid 12 14 16", "boxLengths 6.0 7.0 8.0", "pmeorder 3",
                 "randSeed 42 logFreq 50", "species A mass 2.0 mobility 0.5", "species B",
                 "bond 1 harmonic 1.5 0.0", "potential gaussian A B 5.3 0.7071 ramp 6.0",
                 "potential erf2 A A 0.1 1.0 0.5", "integrator all GJF delt 0.005"]:
        b.command(line)
    d = b.describe()
    assert d["Dim"] == 3 and d["grid"] == [12, 14, 16] and d["pmeorder"] == 3
    assert abs(d["L"][1] - 7.0) < 1e-6 and d["randSeed"] == 42 and d["logFreq"] == 50
    assert d["species"][0] == {"label": "A", "mass": 2.0, "mobility": 0.5}
    assert d["species"][1]["mass"] == 1.0 and d["species"][1]["mobility"] == 1.0
    p0, p1 = d["potentials"]
    assert p0["kind"] == "gaussian" and p0["ramp"] and abs(p0["A_final"] - 6.0) < 1e-9
    assert p1["kind"] == "erf2" and abs(p1["Rp"] - 1.0) < 1e-9 and abs(p1["sigma"] - 0.5) < 1e-9
    (it,) = d["integrators"]           # delt is a float as in ps_integrator.h:34
    assert it["group"] == "all" and it["name"] == "GJF" and abs(it["delt"] - 0.005) < 1e-9
    b.close()


def test_read_data_file(tmp_path):
    s = synth.small_system(seed=1, charges=True)
    scr, data = s.write(str(tmp_path))
    b = tild_b200.Box(0, base_dir=str(tmp_path))
    text = open(scr).read().split("endBox")[0]
    for line in text.splitlines():
        if line.startswith("box"):
            continue
        b.command(line)
    info = b.info()
    assert info.nstot == s.N
    assert abs(info.L[0] - s.L[0]) < 1e-5
    d = b.describe()
    assert d["nstot"] == s.N and d["doCharges"]
    b.close()


def test_endbox_without_gpu_reports_cuda(tmp_path):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    s = synth.small_system(seed=1)
    b = tild_b200.box_from_spec(s, options={"write_files": 0})
    with pytest.raises(tild_b200.TildError) as e:
        b.command("endBox")
    assert e.value.code == 4 and "CUDA" in str(e.value)


@pytest.mark.parametrize("lines,code,msg", [
    (["Dim 3", "foo 1"], 2, "Invalid keyword foo"),
    (["grid 8 8 8"], 2, "Dim must be defined before grid"),
    (["Dim 3", "bond 1 quartic 1 1"], 2, "Bond type not supported"),
    (["Dim 3", "potential bias A 1"], 6, "outside the TILD step"),
    (["Dim 3", "potential morse A B 1"], 2, "not a supported potential"),
    (["Dim 3", "potential wall A w 1.0 1 2.0"], 2, "axis must be x, y, or z"),
    (["Dim 2", "potential wall A z 1.0 1 2.0"], 2, "box is only 2-dimensional"),
    (["Dim 3", "potential wall A z 1.0 2 2.0"], 2, "dirSign must be +1 or -1"),
    (["Dim 3", "potential wall A z 1.0 1 2.0 ramp 3.0"], 2, "ramping applied on an unsupported potential"),
    (["Dim 3", "potential gaussian A B 1.0 0.5 foo"], 2, "Invalid keyword: foo"),
    (["Dim 3", "potential gaussian A B 1.0 0.5 ramp"], 2, "no final prefactor"),
    (["Dim 3", "integrator all VV"], 6, "VV"),
    (["Dim 3", "integrator all XYZ"], 2, "not a valid Integrator"),
    (["Dim 3", "integrator all GJF dt 0.1"], 2, "Invalid keyword in Integrator"),
    (["Dim 3", "molecule grafted 10"], 6, "molecule"),
    (["Dim 3", "molecule linear nmolecs 2 1 4 A"], 2, "rho0 must be defined"),
    (["Dim 3", "readData does_not_exist.data"], 3, "Failed to open"),
    (["Dim 3", "species"], 2, "Missing label for species"),
    (["Dim 3", "pmeorder 7"], 2, "pmeorder"),
])
def test_malformed_scripts_are_rejected(lines, code, msg):
    b = tild_b200.Box(0)
    with pytest.raises(tild_b200.TildError) as e:
        for ln in lines:
            b.command(ln)
    assert e.value.code == code, str(e.value)
    assert msg in str(e.value)
    b.close()


def _box_for(spec, extra=(), q=None):
    b = tild_b200.Box(0, options={"write_files": 0})
    b.command("Dim 3")
    b.command("boxLengths %g %g %g" % tuple(spec.L))
    b.command("grid %d %d %d" % tuple(spec.grid))
    if q is not None:
        b.command("doCharges")
    b.command("species A")
    b.command("species B")
    b.set_particles(spec.x, spec.types, spec.mol, q)
    for e in extra:
        b.command(e)
    return b


def test_endbox_checks_before_gpu():
    s = synth.small_system(seed=3)
    q = np.zeros(s.N, np.float32)
    q[0] = 1.0                                   # net charge 1 -> rejected at endBox
    b = _box_for(s, ["integrator all GJF"], q=q)
    with pytest.raises(tild_b200.TildError) as e:
        b.command("endBox")
    assert e.value.code == 2 and "net charge" in str(e.value)
    s2 = synth.small_system(seed=3)
    s2.types[:] = 0                              # species B has no particles -> size-0 group
    b = _box_for(s2, ["integrator all GJF"])
    with pytest.raises(tild_b200.TildError) as e:
        b.command("endBox")
    assert "size 0" in str(e.value)


def test_bond_errors():
    s = synth.small_system(seed=3)
    b = _box_for(s)
    with pytest.raises(tild_b200.TildError) as e:
        b.set_bonds(np.array([[0, s.N + 5]]))
    assert "out of range" in str(e.value)
    b = _box_for(s)
    with pytest.raises(tild_b200.TildError) as e:
        b.set_bonds(np.array([[0, 1], [0, 2], [0, 3]]))   # MAXBONDS = 2
    assert "MAXBONDS" in str(e.value)


@pytest.mark.parametrize("key,good,bad", [
    ("tile_codes", 8, 3), ("deposit_codes", 16, 4), ("deposit_threads", 128, 48), ("gather_threads", 160, 512),
])
def test_tile_options_checked(key, good, bad):
    """Tile and CTA-size options take their documented ranges (0 = chosen) and refuse the
    rest with TILD_ERR_ARG before any GPU work."""
    b = tild_b200.Box(0)
    b.set_option(key, good)
    b.set_option(key, 0)
    with pytest.raises(tild_b200.TildError) as e:
        b.set_option(key, bad)
    assert e.value.code == 1 and key in str(e.value)
    b.close()


def test_synth_data_round_trip(tmp_path):
    """The synthetic writer's file parses back to the same arrays through the library."""
    s = synth.config_c2(scale=1e-3)
    scr, data = s.write(str(tmp_path))
    assert abs(s.charges.sum()) == 0.0
    b = tild_b200.Box(0, base_dir=str(tmp_path))
    for line in open(scr).read().split("endBox")[0].splitlines()[1:]:
        b.command(line)
    d = b.describe()
    assert d["nstot"] == s.N and d["grid"] == [int(v) for v in s.grid]
    assert d["nBonds"] == 0   # counted at endBox
    b.close()
