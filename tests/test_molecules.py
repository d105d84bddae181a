"""`molecule linear` (PS_Box_moleculeMakers.cu:15-311) against the reference's own build.

tests/golden/molecules_ref.npz holds what the unmodified reference made from
MOLECULE_SCRIPT (tests/golden/make_ref_molecules.py): its positions after set-up and its
init.input.data.  The host part (types, molecule ids, charges, bonds with per-side types,
angles, and the positions as the data file prints them) is compared on the CPU; the
positions themselves must be bit-identical on the GPU (same host RNG, same float
rounding).
"""
import os
import sys

import numpy as np
import pytest

import tild_b200

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from make_ref_molecules import MOLECULE_SCRIPT  # noqa: E402

FIX = os.path.join(os.path.dirname(__file__), "golden", "molecules_ref.npz")
pytestmark = pytest.mark.skipif(not os.path.exists(FIX), reason="no reference molecule fixture")


def sections(text):
    """Atoms / Bonds / Angles rows of a data file as lists of token lists."""
    out, cur = {}, None
    for line in text.splitlines():
        t = line.split()
        if len(t) == 1 and t[0] in ("Atoms", "Bonds", "Angles", "Masses"):
            cur = t[0]
            out[cur] = []
        elif t and cur and t[0][0].isdigit():
            out[cur].append(t)
    return out


def build(tmp_path):
    b = tild_b200.Box(base_dir=str(tmp_path), options={"write_files": 1})
    lines = [ln for ln in MOLECULE_SCRIPT.splitlines()[1:] if ln.strip()]
    for ln in lines[:-1]:
        b.command(ln)
    try:
        b.command("endBox")   # writes init.input.data before the device set-up
        ok = True
    except tild_b200.TildError as e:
        assert e.code == 4, e   # no GPU here: the CUDA error comes after the host part
        ok = False
    return b, ok


def test_host_part_matches_reference(tmp_path):
    z = np.load(FIX)
    b, _ = build(tmp_path)
    b.close()
    ours = sections(open(os.path.join(str(tmp_path), "init.input.data")).read())
    ref = sections(str(z["init_data"]))
    for sec in ("Atoms", "Bonds", "Angles"):
        assert ours[sec] == ref[sec], sec


@pytest.mark.gpu
def test_positions_bit_identical(tmp_path):
    z = np.load(FIX)
    b, ok = build(tmp_path)
    assert ok
    x = b.positions()
    b.close()
    assert np.array_equal(x.view(np.uint32), z["x0"].astype(np.float32).view(np.uint32))
