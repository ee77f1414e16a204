"""CPU pins of the time-stepping oracle (oracle/time_oracle.py): the pump
conserves photons (every absorbed photon excites one ion: sum of rate x N_tot
x h x area = absorbed), and without pump and ASE the excitation decays as
exp(-t / tau)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import legacy_mesh

PUMP = dict(peakIntensity=16e3, radius=2.5, exponent=40.0, centerX=0.0, centerY=0.0, wavelength=940e-9,
            sigmaA=0.8e-20, sigmaE=0.16e-20, retroreflect=True)


def test_pump_conserves_photons():
    from oracle import time_oracle as to

    mesh = legacy_mesh("cylindrical")
    clad = np.zeros(mesh.numberOfPrisms, bool)
    rate, absorbed, incident = to.pump_rate(mesh, mesh.betaVolume, PUMP, clad)
    a = mesh.points[mesh.triangles]
    area = 0.5 * np.abs((a[:, 1, 0] - a[:, 0, 0]) * (a[:, 2, 1] - a[:, 0, 1])
                        - (a[:, 1, 1] - a[:, 0, 1]) * (a[:, 2, 0] - a[:, 0, 0]))
    area = area.astype(np.float32).astype(np.float64)
    ions = (rate.reshape(mesh.numberOfLevels - 1, -1) * mesh.nTot * mesh.thickness * area).sum()
    assert ions == np.float64(absorbed) or abs(ions / absorbed - 1) < 1e-12
    assert 0 < absorbed < incident


def test_decay_is_exponential():
    from oracle import time_oracle as to

    mesh = legacy_mesh("cylindrical")
    hist, _ = to.simulate(mesh, mesh.betaVolume, pump=PUMP,
                          time=dict(timeStep=2e-5, steps=4, pumpSteps=0, aseSteps=0, integrator=0),
                          sigma_ase=(1.1e-21, 2.2e-20))
    np.testing.assert_allclose(hist[1:] / hist[:-1], np.exp(-2e-5 / mesh.crystalTFluo), rtol=1e-9)


@pytest.mark.parametrize("code", range(7))
def test_oracle_integrators_fluorescence_known_answer(code):
    """Pump and ASE off, d beta/dt = -beta/tau: one step multiplies beta by
    each integrator's amplification factor (h = dt/tau)."""
    from haseongpu_b200.configs import disc_small
    from oracle import time_oracle as to

    mesh = disc_small().mesh
    dt = 2e-4
    h = dt / mesh.crystalTFluo
    factor = {0: 1 - h + h**2 / 2 - h**3 / 6 + h**4 / 24, 1: 1 - h, 2: 1 - h + h**2 / 2, 3: 1 - h + h**2 / 2,
              4: 1 - h + h**2 / 2 - h**3 / 6 + h**4 / 24, 5: sum((-h) ** k for k in range(4)), 6: np.exp(-h)}[code]
    pump = dict(peakIntensity=0.0, radius=0.3, exponent=2.0, centerX=0.0, centerY=0.0, wavelength=940e-9,
                sigmaA=7.6e-21, sigmaE=1e-22, retroreflect=True)
    time = dict(timeStep=dt, steps=2, pumpSteps=0, aseSteps=0, integrator=code, implicitIterations=3)
    hist, _ = to.simulate(mesh, mesh.betaVolume, pump=pump, time=time, sigma_ase=(1.1e-21, 2.2e-20))
    np.testing.assert_allclose(hist[-1], mesh.betaVolume * factor**2, rtol=1e-13)
