"""GPU parity of the time-stepped rate equations (hase_simulate) against the
CPU restatement oracle/time_oracle.py.

The device integrates in FP64 like the oracle; they differ by the last bits
of exp / pow on the two sides (pump) and by nothing else, so beta agrees to
~1e-12 relative without ASE.  With ASE the oracle replays the device's phi-ASE
of every solve (phiHistory), and beta agrees to ~1e-9.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import legacy_mesh

pytestmark = pytest.mark.gpu

PUMP = dict(peakIntensity=16e3, radius=2.5, exponent=40.0, centerX=0.0, centerY=0.0, wavelength=940e-9,
            sigmaA=0.8e-20, sigmaE=0.16e-20, retroreflect=True)


def _ctx(mesh, sa, se):
    from haseongpu_b200 import DeviceMesh, build

    build.build_library()
    return DeviceMesh(mesh, sa, se, device=0)


def _cladding_mesh():
    """The true-cladding disc (cladding ring, absorption 5.5 / cm) at 1030 nm."""
    return legacy_mesh("true_cladding", claddingAbsorption=5.5), [5e-21], [1e-20]


def test_pump_and_fluorescence_match_oracle():
    from oracle import time_oracle as to

    mesh, sa, se = _cladding_mesh()
    beta0 = mesh.betaVolume.copy()
    time = dict(timeStep=2e-5, steps=12, pumpSteps=8, aseSteps=0, integrator=0)
    with _ctx(mesh, sa, se) as ctx:
        out = ctx.simulate(pump=PUMP, time=time, minRays=1000, monochromatic=True)
    hist, absorbed = to.simulate(mesh, beta0, pump=PUMP, time=time, sigma_ase=(sa[0], se[0]))
    np.testing.assert_allclose(out["betaVolume"], hist[-1], rtol=1e-11, atol=1e-14)
    gain = ~np.tile(mesh.claddingCellTypes == mesh.claddingNumber, mesh.numberOfLevels - 1)
    np.testing.assert_allclose(out["meanBeta"], hist[:, gain].mean(axis=1), rtol=1e-11)
    np.testing.assert_allclose(out["pumpAbsorbed"], absorbed, rtol=1e-9, atol=1e-15)
    assert out["meanBeta"][8] > out["meanBeta"][0]          # the pump excites
    assert np.all(np.diff(out["meanBeta"][9:]) < 0)         # then the excitation decays
    np.testing.assert_array_equal(out["betaVolume"][~gain], beta0[~gain])  # cladding keeps its beta


def test_decay_without_pump_is_exponential():
    mesh, sa, se = _cladding_mesh()
    time = dict(timeStep=2e-5, steps=5, pumpSteps=0, aseSteps=0, integrator=0)
    with _ctx(mesh, sa, se) as ctx:
        out = ctx.simulate(pump=PUMP, time=time, minRays=1000, monochromatic=True)
    ratio = out["meanBeta"][1:] / out["meanBeta"][:-1]
    np.testing.assert_allclose(ratio, np.exp(-2e-5 / mesh.crystalTFluo), rtol=1e-10)


INTEGRATORS = ["frozen-phi-ase-runge-kutta-4", "explicit-euler", "heun", "midpoint", "runge-kutta-4",
               "implicit-euler", "exponential-euler"]


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_ase_steps_replay_the_oracle(integrator):
    """Every integrator of the reference, with phi-ASE re-solved at the stages
    that re-solve it: the oracle integrates the device's own phi of every
    solve (phiHistory, in order) and reaches the same beta."""
    from haseongpu_b200.simulation import solves_per_step, time_integrator
    from oracle import time_oracle as to

    mesh, sa, se = _cladding_mesh()
    beta0 = mesh.betaVolume.copy()
    time = dict(timeStep=2e-5, steps=3, pumpSteps=3, aseSteps=2, integrator=integrator, implicitIterations=3)
    k = solves_per_step(integrator, 3)
    with _ctx(mesh, sa, se) as ctx:
        out = ctx.simulate(pump=PUMP, time=time, minRays=4000, monochromatic=True, keepPhi=True)
    assert out["phiHistory"].shape == (2 * k, mesh.numberOfSamples) and np.all(out["phiHistory"] > 0)
    otime = dict(time, integrator=time_integrator(integrator))
    hist, _ = to.simulate(mesh, beta0, pump=PUMP, time=otime, sigma_ase=(sa[0], se[0]),
                          phi_history=out["phiHistory"])
    np.testing.assert_allclose(out["betaVolume"], hist[-1], rtol=1e-9, atol=1e-14)
    assert out["raysTraced"] == 2 * k * 4000 * mesh.numberOfSamples
    assert out["meanPhi"][2] == 0.0 and out["meanPhi"][0] > 0
    if k > 1:  # the stage solves saw the stage states: their phi differs from the step-start solve
        assert np.any(out["phiHistory"][1] != out["phiHistory"][0])


@pytest.mark.parametrize("integrator", INTEGRATORS)
def test_fluorescence_decay_known_answer(integrator):
    """Pump and ASE off: d beta/dt = -beta/tau in every gain prism, so one
    step of size h = dt/tau multiplies beta by the integrator's own
    amplification factor -- 1 - h (explicit Euler), 1 - h + h^2/2 (Heun,
    midpoint), the 4-term Taylor sum of e^-h (RK4), sum_{k<=N} (-h)^k (N
    fixed-point iterations of implicit Euler), e^-h (exponential Euler)."""
    from haseongpu_b200.simulation import time_integrator

    mesh, sa, se = _cladding_mesh()
    dt = 2e-4
    h = dt / mesh.crystalTFluo
    code = time_integrator(integrator)
    factor = {0: 1 - h + h**2 / 2 - h**3 / 6 + h**4 / 24, 1: 1 - h, 2: 1 - h + h**2 / 2, 3: 1 - h + h**2 / 2,
              4: 1 - h + h**2 / 2 - h**3 / 6 + h**4 / 24, 5: sum((-h) ** k for k in range(4)), 6: np.exp(-h)}[code]
    time = dict(timeStep=dt, steps=3, pumpSteps=0, aseSteps=0, integrator=integrator, implicitIterations=3)
    with _ctx(mesh, sa, se) as ctx:
        out = ctx.simulate(pump=PUMP, time=time, minRays=1000, monochromatic=True)
    gain = mesh.betaVolume > 0
    np.testing.assert_allclose(out["betaVolume"][gain], mesh.betaVolume[gain] * factor**3, rtol=1e-12)


def test_learned_proposal_in_the_time_loop():
    from haseongpu_b200.proposal import ProposalNet

    mesh, sa, se = _cladding_mesh()
    time = dict(timeStep=2e-5, steps=2, pumpSteps=2, aseSteps=2, integrator=0)
    with _ctx(mesh, sa, se) as ctx, ProposalNet(seed=3) as net:
        out = ctx.simulate(pump=PUMP, time=time, net=net, fallbackVariance=1e9, minRays=4000, monochromatic=True)
    assert np.all(np.isfinite(out["betaVolume"])) and out["fallbackSamples"] == 0
    assert out["meanPhi"][0] > 0 and out["meanBeta"][2] > out["meanBeta"][0]


def _twin(mesh, sa, se):
    from haseongpu_b200 import TetDeviceMesh, TetMesh

    return TetDeviceMesh(TetMesh.fromPrismMesh(mesh), sa, se, device=0)


def test_forward_driver_without_ase_equals_the_backward_driver():
    mesh, sa, se = _cladding_mesh()
    time = dict(timeStep=2e-5, steps=6, pumpSteps=4, aseSteps=0, integrator=0)
    with _ctx(mesh, sa, se) as a, _ctx(mesh, sa, se) as b, _twin(mesh, sa, se) as twin:
        back = a.simulate(pump=PUMP, time=time, minRays=1000, monochromatic=True)
        fwd = b.simulate_forward(twin, pump=PUMP, time=time, forwardRayCount=10000, monochromatic=True)
    np.testing.assert_array_equal(fwd["betaVolume"], back["betaVolume"])
    np.testing.assert_allclose(fwd["pumpAbsorbed"], back["pumpAbsorbed"], rtol=1e-12)  # FP64 atomic sums


@pytest.mark.parametrize("integrator", ["frozen-phi-ase-runge-kutta-4", "explicit-euler", "heun",
                                        "runge-kutta-4", "exponential-euler"])
def test_forward_ase_steps_replay_the_oracle(integrator):
    """The oracle replays the forward driver's per-prism phi (volume-weighted
    means of the twin's cells, every solve) through the same rate equations."""
    from haseongpu_b200.simulation import solves_per_step, time_integrator
    from oracle import time_oracle as to

    mesh, sa, se = _cladding_mesh()
    beta0 = mesh.betaVolume.copy()
    time = dict(timeStep=2e-5, steps=3, pumpSteps=3, aseSteps=2, integrator=integrator)
    k = solves_per_step(integrator)
    with _ctx(mesh, sa, se) as ctx, _twin(mesh, sa, se) as twin:
        out = ctx.simulate_forward(twin, pump=PUMP, time=time, forwardRayCount=400_000, monochromatic=True,
                                   keepPhi=True)
    assert out["phiHistory"].shape == (2 * k, mesh.numberOfPrisms)
    assert out["raysTraced"] == 2 * k * 400_000 and out["meanPhi"][0] > 0 and out["meanPhi"][2] == 0.0
    hist, _ = to.simulate(mesh, beta0, pump=PUMP, time=dict(time, integrator=time_integrator(integrator)),
                          sigma_ase=(sa[0], se[0]), phi_prism_history=out["phiHistory"])
    np.testing.assert_allclose(out["betaVolume"], hist[-1], rtol=1e-9, atol=1e-14)


def test_forward_and_backward_ase_agree_on_the_mean_flux():
    """The two methods estimate the same ASE flux: the gain-prism mean of phi
    of the first step agrees to a few percent."""
    mesh, sa, se = _cladding_mesh()
    time = dict(timeStep=2e-5, steps=1, pumpSteps=1, aseSteps=1, integrator=0)
    with _ctx(mesh, sa, se) as a, _ctx(mesh, sa, se) as b, _twin(mesh, sa, se) as twin:
        back = a.simulate(pump=PUMP, time=time, minRays=20000, monochromatic=True, keepPhi=True)
        fwd = b.simulate_forward(twin, pump=PUMP, time=time, forwardRayCount=4_000_000, monochromatic=True,
                                 keepPhi=True)
    from oracle import time_oracle as to

    gain = ~np.tile(mesh.claddingCellTypes == mesh.claddingNumber, mesh.numberOfLevels - 1)
    pb = to.prism_phi(mesh, back["phiHistory"][0])
    pf = fwd["phiHistory"][0]
    assert pf[gain].mean() == pytest.approx(pb[gain].mean(), rel=0.05)
    np.testing.assert_allclose(fwd["betaVolume"][gain].mean(), back["betaVolume"][gain].mean(), rtol=1e-3)
