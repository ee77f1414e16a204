"""Seeded synthetic gain media for the benchmark workloads.

No public dataset is involved: every medium is generated here from a fixed
master seed (20261203) with one ``numpy.random.SeedSequence`` child per
workload.

disc_small   ~550 points on 13 jittered concentric rings of a 1 cm disc,
             Delaunay (~1,000 triangles), 10 levels over 0.7 cm (9 prism
             layers); beta = 0.05 + 0.25 exp(-r^2/(0.4 cm)^2) exp(-z/0.5 cm)
             at each prism centre; N_tot = 1.38e20 cm^-3; one wavelength,
             sigma_e = 2.2e-20, sigma_a = 1.1e-21 cm^2; no reflections;
             rays 1e5 -> 1e6 per sample, relative-error threshold 0.005.
disc_poly    ~2,600 points on 29 rings (~5,100 triangles) x 20 levels, the
             same beta profile x (1 + U(-0.05, 0.05)) noise, 16 wavelength
             pairs from two Lorentzians (peaks 1030 / 940 nm) scaled to
             1e-21..3e-20 cm^2, reflectivity 0.3 bottom / 0.9 top with
             refractive index 1.83 inside / 1.0 outside (total internal
             reflection above the critical angle), order <= 2; rays
             1e5 -> 1e7, threshold 0.001.
media64      64 independent gain media (config 3): per medium a seeded
             triangle count log-uniform in 200..20,000 (ring count chosen
             to match), levels uniform in 5..40, radius U(0.5, 3) cm,
             thickness U(0.3, 2) cm, Gaussian-pump beta with seeded waist
             U(0.3, 0.7) x radius, depth U(0.5, 1.5) x thickness and peak
             U(0.15, 0.35), 1..8 wavelengths (one pair: the disc_small pair;
             more: the two-Lorentzian spectrum); rays 1e4 -> 1e7 per sample,
             threshold 0.001.
pulse        the pump-pulse time series (config 5): ~10,000 points on 56
             jittered rings of a 1 cm disc (~20,000 triangles) x 30 levels
             over 0.7 cm, 8 wavelength pairs of the two-Lorentzian spectrum,
             reflectivity 0.3 bottom / 0.9 top with refractive index 1.83
             inside / 1.0 outside; beta starts at 0 and a 1 ms rectangular
             pump (super-Gaussian, radius 0.6 cm, order 40, 16 kW/cm^2 at
             940 nm, sigma_a 0.8e-20 / sigma_e 0.16e-20 cm^2, retro-reflected)
             drives it over 50 steps of 20 us.
The fluorescence lifetime is 9.41e-4 s (the reference example media,
example/laserPumpCladdingApi.py:241); it only scales phi.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .mesh import PrismMesh, delaunay_triangles, disc_points, gaussian_pump_beta, point_beta
from .spectra import CrossSectionData, two_lorentzian_spectrum

MASTER_SEED = 20261203
TAU = 9.41e-4


@dataclass
class Workload:
    name: str
    mesh: PrismMesh
    spectra: CrossSectionData
    minRays: int
    maxRays: int
    threshold: float
    useReflections: bool
    monochromatic: bool
    adaptiveSteps: int = 4


def _rng(index: int) -> np.random.Generator:
    return np.random.default_rng(np.random.SeedSequence(MASTER_SEED).spawn(8)[index])


def disc_small() -> Workload:
    rng = _rng(0)
    pts = disc_points(1.0, 13, rng)
    tri = delaunay_triangles(pts)
    levels, thickness = 10, 0.7 / 9
    mesh = PrismMesh(points=pts, triangles=tri, numberOfLevels=levels, thickness=thickness,
                     betaVolume=gaussian_pump_beta(pts, tri, levels, thickness), nTot=1.38e20, crystalTFluo=TAU,
                     betaCells=point_beta(pts, levels, thickness), name="disc_small")
    spectra = CrossSectionData.monochromatic(wavelength=1030e-9, crossSectionAbsorption=1.1e-21,
                                             crossSectionEmission=2.2e-20)
    return Workload("disc_small", mesh, spectra, 100_000, 1_000_000, 0.005, False, True)


def disc_poly() -> Workload:
    rng = _rng(1)
    pts = disc_points(1.0, 29, rng)
    tri = delaunay_triangles(pts)
    levels, thickness = 20, 0.7 / 19
    beta = gaussian_pump_beta(pts, tri, levels, thickness)
    beta *= 1.0 + rng.uniform(-0.05, 0.05, beta.size)
    T = tri.shape[0]
    mesh = PrismMesh(points=pts, triangles=tri, numberOfLevels=levels, thickness=thickness, betaVolume=beta,
                     nTot=1.38e20, crystalTFluo=TAU, betaCells=point_beta(pts, levels, thickness),
                     reflectivities=np.tile([0.3, 0.9], (T, 1)), refractiveIndices=[1.83, 1.0, 1.83, 1.0],
                     name="disc_poly")
    return Workload("disc_poly", mesh, two_lorentzian_spectrum(16), 100_000, 10_000_000, 0.001, True, False)


@dataclass
class Medium:
    mesh: PrismMesh
    spectra: CrossSectionData
    wavelengths: int


@dataclass
class MediaWorkload:
    name: str
    media: list
    minRays: int
    maxRays: int
    threshold: float
    adaptiveSteps: int = 6


def batch_medium(rng: np.random.Generator, index: int) -> Medium:
    """One seeded gain medium of the batched-media workload."""
    target_t = float(np.exp(rng.uniform(np.log(200.0), np.log(20000.0))))
    rings = max(3, int(round(np.sqrt(target_t / 6.3))))
    levels = int(rng.integers(5, 41))
    radius = float(rng.uniform(0.5, 3.0))
    height = float(rng.uniform(0.3, 2.0))
    waist = float(rng.uniform(0.3, 0.7)) * radius
    depth = float(rng.uniform(0.5, 1.5)) * height
    peak = float(rng.uniform(0.15, 0.35))
    nl = int(rng.integers(1, 9))
    pts = disc_points(radius, rings, rng)
    tri = delaunay_triangles(pts)
    h = height / (levels - 1)
    mesh = PrismMesh(points=pts, triangles=tri, numberOfLevels=levels, thickness=h,
                     betaVolume=gaussian_pump_beta(pts, tri, levels, h, waist=waist, depth=depth, peak=peak),
                     nTot=1.38e20, crystalTFluo=TAU,
                     betaCells=point_beta(pts, levels, h, waist=waist, depth=depth, peak=peak),
                     name=f"medium{index}")
    if nl == 1:
        spectra = CrossSectionData.monochromatic(wavelength=1030e-9, crossSectionAbsorption=1.1e-21,
                                                 crossSectionEmission=2.2e-20)
    else:
        spectra = two_lorentzian_spectrum(nl)
    return Medium(mesh, spectra, nl)


def media64(count: int = 64) -> MediaWorkload:
    rng = _rng(2)
    return MediaWorkload("media64", [batch_medium(rng, i) for i in range(count)], 10_000, 10_000_000, 0.001)


def media_training(count: int = 24, max_triangles: int = 3000) -> list:
    """Training media for a proposal network that serves the media64 family:
    the same generator on its own seed, media above ``max_triangles``
    skipped (the logged training rows grow with samples x prisms)."""
    rng = _rng(3)
    out = []
    while len(out) < count:
        m = batch_medium(rng, len(out))
        if m.mesh.numberOfTriangles <= max_triangles:
            out.append(m)
    return out


@dataclass
class PulseWorkload:
    name: str
    mesh: PrismMesh
    spectra: CrossSectionData
    pump: dict
    time: dict


def pulse() -> PulseWorkload:
    rng = _rng(4)
    pts = disc_points(1.0, 56, rng)
    tri = delaunay_triangles(pts)
    levels, thickness = 30, 0.7 / 29
    T = tri.shape[0]
    P = T * (levels - 1)
    mesh = PrismMesh(points=pts, triangles=tri, numberOfLevels=levels, thickness=thickness, betaVolume=np.zeros(P),
                     nTot=1.38e20, crystalTFluo=TAU, betaCells=np.zeros(pts.shape[0] * levels),
                     reflectivities=np.tile([0.3, 0.9], (T, 1)), refractiveIndices=[1.83, 1.0, 1.83, 1.0],
                     name="pulse")
    pump = dict(peakIntensity=16e3, radius=0.6, exponent=40.0, centerX=0.0, centerY=0.0, wavelength=940e-9,
                sigmaA=0.8e-20, sigmaE=0.16e-20, retroreflect=True)
    time = dict(timeStep=20e-6, steps=50, pumpSteps=50, aseSteps=50, integrator=0)
    return PulseWorkload("pulse", mesh, two_lorentzian_spectrum(8), pump, time)


WORKLOADS = {"disc_small": disc_small, "disc_poly": disc_poly}
