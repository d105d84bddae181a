import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "matilda.ft_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def spec_to_system(spec, maxb=2, **kw):
    """synth.SystemSpec -> oracle.System."""
    import oracle
    nb, partner, btype = spec.partner_lists(maxb)
    D = spec.dim
    return oracle.System(
        Dim=D, L=np.asarray(spec.L[:D], np.float32), Nx=np.asarray(spec.grid[:D], np.int32),
        order=spec.order, x=np.asarray(spec.x[:, :D], np.float32), types=spec.types,
        mass=np.asarray(spec.masses, np.float32), mobility=np.asarray(spec.mobility, np.float32),
        species=spec.species, charges=spec.charges, nb=nb, partner=partner, btype=btype,
        bond_k=np.array([spec.bond_k], np.float32), bond_req=np.array([spec.bond_req], np.float32),
        bond_style=np.array([0], np.int32), potentials=spec.potentials, delt=spec.delt,
        integrator=spec.integrator, angles=spec.angles if len(spec.angles) else None,
        angle_types=spec.angle_types,
        angle_k=np.array([a["k"] for a in spec.angle_params], np.float32).astype(np.float64),
        angle_theq=np.array([np.float32(a.get("theta", 0.0) * (np.pi / 180.0)) for a in spec.angle_params],
                            np.float64),
        angle_style=np.array([0 if a["style"] == "wlc" else 1 for a in spec.angle_params], np.int32), **kw)


def force_error(f, fref, tol=None):
    """max_p |f_p - fref_p| / max(|fref_p|, f_rms) (the per-particle metric of the tests);
    with per-particle tolerances tol, the largest error as a multiple of its tolerance."""
    fref = np.asarray(fref, np.float64)
    f = np.asarray(f, np.float64)
    mag = np.linalg.norm(fref, axis=1)
    rms = np.sqrt(np.mean(mag ** 2))
    den = np.maximum(mag, rms)
    err = np.linalg.norm(f - fref, axis=1) / den
    return float(np.max(err if tol is None else err / tol))


def angle_force_tolerance(sysm, base):
    """Per-particle force tolerance: base, raised for the three particles of an angle by the
    FP32 conditioning of its force, 2^-21 / sin^2(theta): cos(theta) carries a few ulps of
    rounding (about six roundings in the dot product and the norms), and the force's
    1/sqrt(1 - cos^2) turns them into a relative error of up to ~6 * 2^-24 / sin^2(theta),
    in any FP32 evaluation (the reference's included; a 0.4-degree bend gives ~3e-3)."""
    tol = np.full(sysm.N, float(base))
    if getattr(sysm, "angles", None) is None or len(sysm.angles) == 0:
        return tol
    x = np.asarray(sysm.x, np.float64)
    L = np.asarray(sysm.L, np.float64)[: x.shape[1]]
    for tri in np.asarray(sysm.angles):
        i, j, k = (int(v) for v in tri)
        rij = x[i] - x[j]
        rkj = x[k] - x[j]
        rij -= L * np.round(rij / L)
        rkj -= L * np.round(rkj / L)
        c = rij @ rkj / (np.linalg.norm(rij) * np.linalg.norm(rkj))
        t = base + 2.0 ** -21 / max(1.0 - c * c, 1e-12)
        for p in (i, j, k):
            tol[p] = max(tol[p], t)
    return tol


@pytest.fixture(scope="session")
def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
