"""Absorption / emission spectra and their resampling.

``CrossSectionData`` mirrors the reference's spectral container
(pyInclude/laser.py:183-260: wavelengthsAbsorption, crossSectionAbsorption,
wavelengthsEmission, crossSectionEmission, resolution, ``monochromatic``,
``fromDirectory``).  ``interpolate_linear`` restates the reference's
``hase::utils::interpolateLinear`` (src/utils/interpolation.cpp): resample y(x)
onto ``n`` equidistant x over [x0, x_last], last value pinned to y[-1].  As in
the reference parser (src/openpmd/OpenPmdParser.cpp:1370-1389) absorption and
emission are resampled independently to ``resolution`` samples and paired by
index.
"""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np


def interpolate_linear(y, x, n: int) -> np.ndarray:
    y = np.asarray(y, np.float64).ravel()
    x = np.asarray(x, np.float64).ravel()
    if x.size == 0 or x.size != y.size:
        raise ValueError("x and y must be non-empty and of equal length")
    if n < y.size:
        raise ValueError("resolution must be >= the number of input samples")
    if n == 0:
        return np.empty(0)
    if y.size == 1:
        return np.full(n, y[0])
    if np.any(np.diff(x) <= 0):
        raise ValueError("x must be strictly increasing")
    xi = x[0] + (np.arange(n, dtype=np.float64) * (x[-1] - x[0])) / float(n - 1)
    # segment i covers [x[i], x[i+1]); points at or beyond x[-1] keep 0 until pinned below
    seg = np.searchsorted(x, xi, side="right") - 1
    out = np.zeros(n)
    valid = seg < x.size - 1
    s = seg[valid]
    m = (y[s + 1] - y[s]) / (x[s + 1] - x[s])
    b = y[s] - m * x[s]
    out[valid] = b + m * xi[valid]
    out[-1] = y[-1]
    return out


@dataclass
class CrossSectionData:
    wavelengthsAbsorption: np.ndarray
    crossSectionAbsorption: np.ndarray
    wavelengthsEmission: np.ndarray
    crossSectionEmission: np.ndarray
    resolution: int = 1

    def __post_init__(self):
        for name in ("wavelengthsAbsorption", "crossSectionAbsorption", "wavelengthsEmission",
                     "crossSectionEmission"):
            setattr(self, name, np.asarray(getattr(self, name), np.float64).reshape(-1))
        self.resolution = int(self.resolution)
        if self.wavelengthsAbsorption.size != self.crossSectionAbsorption.size:
            raise ValueError("wavelengthsAbsorption and crossSectionAbsorption must have the same length")
        if self.wavelengthsEmission.size != self.crossSectionEmission.size:
            raise ValueError("wavelengthsEmission and crossSectionEmission must have the same length")
        if self.resolution < 1:
            raise ValueError("resolution must be positive")

    @classmethod
    def monochromatic(cls, *, wavelength, crossSectionAbsorption, crossSectionEmission):
        return cls([wavelength], [crossSectionAbsorption], [wavelength], [crossSectionEmission], 1)

    @classmethod
    def fromDirectory(cls, path, resolution=1000):
        root = Path(path)
        return cls(np.loadtxt(root / "lambda_a.txt"), np.loadtxt(root / "sigma_a.txt"),
                   np.loadtxt(root / "lambda_e.txt"), np.loadtxt(root / "sigma_e.txt"), resolution)

    @property
    def maxSigmaA(self) -> float:
        return float(np.max(self.crossSectionAbsorption))

    @property
    def maxSigmaE(self) -> float:
        return float(np.max(self.crossSectionEmission))

    def resampled(self, monochromatic: bool = False):
        """(sigmaA, sigmaE) as handed to the device: first pair only when
        ``monochromatic`` (the legacy parser's reduction), else both spectra
        resampled to ``resolution`` samples."""
        sa, se = self.crossSectionAbsorption, self.crossSectionEmission
        if monochromatic:
            return sa[:1].copy(), se[:1].copy()
        n = max(self.resolution, sa.size, se.size)
        if sa.size == se.size == n:
            return sa.copy(), se.copy()
        return (interpolate_linear(sa, self.wavelengthsAbsorption, n),
                interpolate_linear(se, self.wavelengthsEmission, n))


def two_lorentzian_spectrum(n: int, peaks=(1030.0, 940.0), widths=(6.0, 12.0), lo=1e-21, hi=3e-20,
                            span=(900.0, 1070.0)) -> CrossSectionData:
    """Seedless synthetic spectrum: emission = sum of two Lorentzians (peak near
    ``peaks``), absorption = the same with the weights swapped, both scaled to
    [lo, hi] cm^2 and sampled at ``n`` wavelengths over ``span`` nm."""
    lam = np.linspace(span[0], span[1], n)

    def lor(c, w):
        return 1.0 / (1.0 + ((lam - c) / w) ** 2)

    def scale(v):
        v = (v - v.min()) / (v.max() - v.min())
        return lo + (hi - lo) * v

    emission = scale(1.0 * lor(peaks[0], widths[0]) + 0.35 * lor(peaks[1], widths[1]))
    absorption = scale(0.25 * lor(peaks[0], widths[0]) + 1.0 * lor(peaks[1], widths[1]))
    return CrossSectionData(lam, absorption, lam, emission, resolution=n)
