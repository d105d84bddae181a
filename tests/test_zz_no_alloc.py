"""The allocation-free density read-back against the allocating one, on the GPU.

tild_box_get_density_noalloc is for callers that cannot allocate device memory (their
pool allocator holds the device's memory, or a cudaFree would synchronise streams they
keep busy); it takes its device scratch from one static device array instead of
cudaMalloc.  It must return the density tild_box_get_density returns on two calls in a
row (the accumulator in the static array keeps the previous call's contents, so every
call has to clear it), and it must refuse a box whose scratch does not fit.  Tolerance:
|drho| <= 1e-6 * max|rho| (the two entry points deposit with FP32 atomics in different
orders).

The file name sorts last so that a run stopping at the first failure has run every other
test before this one.
"""
import numpy as np
import pytest

import tild_b200
from tild_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-6


def make_box(spec, **opts):
    o = {"write_files": 0}
    o.update(opts)
    b = tild_b200.box_from_spec(spec, options=o)
    b.command("endBox")
    return b


def close(a, b):
    return np.abs(a - b).max() <= TOL * max(np.abs(b).max(), 1e-30)


@pytest.mark.parametrize("charges", [False, True])
def test_noalloc_density_matches_allocating(charges):
    spec = synth.small_system(seed=31, order=3, charges=charges, grid=(15, 12, 18))
    with make_box(spec, sort_interval=3) as b:
        b.step(7)   # particles re-sorted: slots differ from particle ids
        groups = [("all", False), ("A", False), ("B", False)]
        if charges:
            groups.append(("charges", True))
        for name, qch in groups:
            ref = b.density(name, charge=qch)
            got1 = b.density_noalloc(name, charge=qch)
            got2 = b.density_noalloc(name, charge=qch)
            assert np.abs(ref).max() > 0
            assert close(got1, ref), name
            assert close(got2, ref), name


def test_noalloc_density_rejects_oversize_grid():
    spec = synth.small_system(seed=32, order=1, grid=(192, 192, 192), L=20.0)
    with make_box(spec) as b:
        need = 4 * (192 ** 3 + b.N + b.N)
        assert need > tild_b200.NOALLOC_SCRATCH_BYTES
        with pytest.raises(tild_b200.TildError, match="static scratch"):
            b.density_noalloc("all")
        # the box stays usable
        assert np.isfinite(b.density("all")).all()
