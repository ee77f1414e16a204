"""Shared fixtures.  GPU tests carry ``@pytest.mark.gpu``; everything else runs on CPU."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as _oracle

    _oracle.build()
    return _oracle


@pytest.fixture(scope="session")
def native():
    from haseongpu_b200 import _native, build

    build.build_library()
    return _native


def legacy_mesh(name, claddingAbsorption=None):
    from haseongpu_b200 import PrismMesh

    return PrismMesh.fromLegacyFixture(GOLDEN / f"legacy_{name}.npz", claddingAbsorption=claddingAbsorption)


def legacy_spectrum(name):
    d = np.load(GOLDEN / f"legacy_{name}.npz")
    return [float(d["sigmaA"])], [float(d["sigmaE"])]


def analytic_phi(mesh, sample_xyz, beta, g, nTot, tau, n_mu=512, n_phi=512):
    """Quadrature known answer for uniform beta and gain g in a convex extruded polygon:

    phi(s) = N_tot beta / (4 pi tau) * Int_{S^2} expm1(g L(Omega)) / g dOmega,

    L the distance from s to the medium boundary along Omega (the reference's
    sphere known answer, tests/python/phiAse/test_analyticalSphere.py:19-31,
    generalised to any convex prism stack)."""
    from scipy.spatial import ConvexHull

    pts = mesh.points
    hull = pts[ConvexHull(pts).vertices]  # counter-clockwise
    edges = np.roll(hull, -1, axis=0) - hull
    normals = np.column_stack([edges[:, 1], -edges[:, 0]])
    normals /= np.linalg.norm(normals, axis=1, keepdims=True)
    c = (normals * hull).sum(axis=1)
    H = mesh.thickness * (mesh.numberOfLevels - 1)
    mu, wmu = np.polynomial.legendre.leggauss(n_mu)
    phi = (np.arange(n_phi) + 0.5) * 2 * np.pi / n_phi
    M, PHI = np.meshgrid(mu, phi, indexing="ij")
    sin_t = np.sqrt(1 - M ** 2)
    dx, dy = sin_t * np.cos(PHI), sin_t * np.sin(PHI)
    x, y, z = sample_xyz
    L = np.full(M.shape, np.inf)
    for n, ce in zip(normals, c):
        den = n[0] * dx + n[1] * dy
        num = ce - (n[0] * x + n[1] * y)
        with np.errstate(divide="ignore", invalid="ignore"):
            t = np.where(den > 1e-15, np.maximum(num, 0.0) / den, np.inf)
        L = np.minimum(L, t)
    with np.errstate(divide="ignore"):
        tz = np.where(M > 0, (H - z) / M, np.where(M < 0, -z / M, np.inf))
    L = np.minimum(L, tz)
    f = np.expm1(g * L) / g if g != 0 else L
    integral = (f * wmu[:, None]).sum() * (2 * np.pi / n_phi)
    return nTot * beta / (4 * np.pi * tau) * integral
