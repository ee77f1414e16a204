"""CPU: the polychromatic estimate's reported error is its error.

Rays are ordered by prism (the ray map is a prefix over the weight row), so a
wavelength drawn from the ray index in contiguous strata gives whole regions
of the medium one wavelength per pass, and the rays' sample variance misses
the between-wavelength part.  Each ray now averages its gain over the whole
spectrum (its walk's path integrals give every wavelength's exponent), so
the rays are independent again.  Check: over eight seeds, the spread of each
sample's estimate stays within its reported relative error (16 wavelengths,
reflections, fixed importance weights, 40,000 rays)."""

from __future__ import annotations

import numpy as np


def test_polychromatic_seed_spread_within_reported_error(oracle):
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    sa, se = w.spectra.resampled()
    s0, ns = 3000, 4
    W = np.stack([oracle.importance(w.mesh, (sa, se), s, 5) for s in range(s0, s0 + ns)]).astype(np.float32)
    est, rse = [], []
    for seed in range(1, 9):
        r = oracle.phi_ase(w.mesh, (sa, se), minRays=40000, useReflections=True, seed=seed, minSample=s0,
                           maxSample=s0 + ns - 1, weights=W)
        est.append(r["phiAse"])
        rse.append(r["mse"])
    est, rse = np.array(est), np.array(rse)
    spread = est.std(axis=0, ddof=1) / est.mean(axis=0)
    # eight seeds: the sample standard deviation is within ~1.6x of sigma at 90 %
    assert np.all(spread < 1.6 * np.median(rse, axis=0)), (spread, np.median(rse, axis=0))


def test_spectral_mean_is_the_mean_of_monochromatic_estimates(oracle):
    """The oracle's polychromatic estimate (each ray's gain averaged over the
    16 wavelengths from its path integrals) agrees with the mean of the 16
    monochromatic estimates within the combined error (same importance
    weights, independent seeds)."""
    from haseongpu_b200.configs import disc_poly

    w = disc_poly()
    sa, se = w.spectra.resampled()
    s0, ns = 3000, 3
    W = np.stack([oracle.importance(w.mesh, (sa, se), s, 5) for s in range(s0, s0 + ns)]).astype(np.float32)
    kw = dict(minRays=20000, useReflections=True, minSample=s0, maxSample=s0 + ns - 1, weights=W)
    poly = oracle.phi_ase(w.mesh, (sa, se), seed=1, **kw)
    phis, var = [], []
    for lam in range(len(sa)):
        r = oracle.phi_ase(w.mesh, ([float(sa[lam])], [float(se[lam])]), seed=100 + lam, **kw)
        phis.append(r["phiAse"])
        var.append((r["mse"] * r["phiAse"]) ** 2)
    mean = np.mean(phis, axis=0)
    sigma = np.hypot(poly["mse"] * poly["phiAse"], np.sqrt(np.sum(var, axis=0)) / len(sa))
    z = (poly["phiAse"] - mean) / sigma
    assert np.all(np.abs(z) < 4.0), z
