"""The benchmarked workload at full size: the polyelectrolyte coacervate of 2,097,152
particles (8,000 + 8,000 chains of 32 charged beads, 512,000 counterions, neutral solvent)
on a 192^3 grid with a Gaussian excluded volume (all, all) and smeared charges (lB 1.0,
sigma 0.5), pmeorder 3.  FP32 deposit, FFT and interpolation against the FP64 oracle
(PS_Box::forces, PS_Box.cu:240-278, with the charges' CalcForces,
ps_potentialCharges.cu:125-164):

  * forces at step 0, per particle |df_p| / max(|f_p|, f_rms) <= 1e-5 for every particle;
  * the Gaussian pair energy and the charge energy (1/2 gvol sum rhoq phi,
    ps_potentialCharges.cu:71-118): relative 1e-5; the bond energy: relative 1e-6.
"""
import numpy as np
import pytest

import oracle
import tild_b200
from conftest import spec_to_system
from tild_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2_reference():
    spec = synth.config_c2()
    assert spec.N == 2097152 and list(spec.grid) == [192, 192, 192]
    sysm = spec_to_system(spec)
    fref, inter = oracle.forces(sysm, prec=64)
    return spec, sysm, fref, inter


# the density rule's deposit tiles (8 bricks: int32 boxes at 2^24 per unit weight), and the
# 32- and 64-brick tiles the autotuner picks on this workload (about 600 and 1,200 particles
# each: 2^23 and 2^22, FP32 for the rare tile past four times the count bound)
@pytest.mark.parametrize("deposit_codes,deposit_threads", [(0, 0), (32, 0), (64, 512)])
def test_c2_forces_and_energies_match_the_fp64_oracle(c2_reference, deposit_codes, deposit_threads):
    spec, sysm, fref, inter = c2_reference
    opts = {"write_files": 0, "deposit_codes": deposit_codes, "deposit_threads": deposit_threads}
    with tild_b200.box_from_spec(spec, options=opts) as b:
        b.command("endBox")
        f = b.forces()
        th = b.thermo()
    mag = np.linalg.norm(fref, axis=1)
    den = np.maximum(mag, np.sqrt(np.mean(mag ** 2)))
    err = np.linalg.norm(f - fref, axis=1) / den
    print("c2 (deposit_codes %d) force error percentiles 50/99/99.9/max:" % deposit_codes,
          np.percentile(err, [50, 99, 99.9]), err.max())
    assert err.max() <= 1e-5
    pe = oracle.pair_energies(sysm, inter["dens"])
    assert len(th["potentials"]) == 2
    for e, r in zip(th["potentials"], pe):
        assert abs(e - r) <= 1e-5 * abs(r), (e, r)
    ub, _ = oracle.bond_energy(sysm)
    assert abs(th["Ubond"] - ub) <= 1e-6 * abs(ub)
