"""CPU restatement of the time-stepped rate equations of hase_simulate
(TEST INFRASTRUCTURE ONLY: the product never imports this file).

Per gain prism (include/kernels/derivativeComposition.hpp:27-93):
    d beta/dt = pump(beta) - [beta (sE + sA) - sA] Phi - beta / tau,
cladding prisms keep their beta.  Phi of a prism is the mean phi-ASE of its
six vertices (float32, as the device).  Pump: a collimated super-Gaussian
beam entering the bottom along +z, optionally retro-reflected at the top;
per triangle column Beer-Lambert with g_p = N_tot [beta (sA_p + sE_p) - sA_p]
per layer, absorbed photons / (N_tot h) (cladding prisms attenuate with
claddingAbsorption and gain nothing).  Integration: the reference's seven
integrators in its stage order (include/core/timeSteppedSimulation.hpp:321-415)
and update forms (include/kernels/timeIntegrationUpdateKernels.hpp:21-105):
frozen-phi-ase-runge-kutta-4 (0), explicit-euler (1), heun (2), midpoint (3),
runge-kutta-4 (4), implicit-euler (5, fixed-point iterations) and
exponential-euler (6); beta clipped to [0, 1] after every step's update as the
reference's ClipBeta.  Integrators 2-5 re-solve phi-ASE at every stage they
evaluate; the phi-ASE of each solve comes from the caller (the device's
phiHistory, one entry per solve in order), so both integrate the same ASE
terms.
"""

from __future__ import annotations

import numpy as np

PLANCK = 6.62607015e-34
LIGHT = 2.99792458e8


def pump_rate(mesh, beta, pump, clad):
    """d beta / dt from the pump, [P]; and absorbed photons / s."""
    T, L = mesh.numberOfTriangles, mesh.numberOfLevels - 1
    cen = mesh.points[mesh.triangles].mean(axis=1)
    a = mesh.points[mesh.triangles]
    area = 0.5 * np.abs((a[:, 1, 0] - a[:, 0, 0]) * (a[:, 2, 1] - a[:, 0, 1])
                        - (a[:, 1, 1] - a[:, 0, 1]) * (a[:, 2, 0] - a[:, 0, 0]))
    area = area.astype(np.float32).astype(np.float64)
    cen = cen.astype(np.float32).astype(np.float64)
    flux0 = pump["peakIntensity"] / (PLANCK * LIGHT / pump["wavelength"])
    r = np.hypot(cen[:, 0] - pump["centerX"], cen[:, 1] - pump["centerY"])
    phi = flux0 * np.exp(-(r / pump["radius"]) ** pump["exponent"])
    phi0 = phi.copy()
    h, nTot = mesh.thickness, mesh.nTot
    b = np.asarray(beta, np.float64).reshape(L, T)
    cl = np.asarray(clad, bool).reshape(L, T)
    rate = np.zeros((L, T))
    order = list(range(L)) + (list(range(L - 1, -1, -1)) if pump["retroreflect"] else [])
    for l in order:
        g = np.where(cl[l], -mesh.claddingAbsorption, nTot * (b[l] * (pump["sigmaA"] + pump["sigmaE"]) - pump["sigmaA"]))
        out = phi * np.exp(g * h)
        rate[l] += np.where(cl[l], 0.0, (phi - out) / (nTot * h))
        phi = out
    return rate.ravel(), float(((phi0 - phi) * area).sum()), float((phi0 * area).sum())


def prism_phi(mesh, phi_samples):
    T, L, Np = mesh.numberOfTriangles, mesh.numberOfLevels - 1, mesh.numberOfPoints
    ps = np.asarray(phi_samples, np.float32).reshape(mesh.numberOfLevels, Np)
    tri = mesh.triangles.astype(np.int64)
    out = np.empty((L, T), np.float32)
    for l in range(L):
        a, b = ps[l][tri], ps[l + 1][tri]
        s = a[:, 0] + a[:, 1] + a[:, 2] + b[:, 0] + b[:, 1] + b[:, 2]
        out[l] = s * np.float32(1.0 / 6.0)
    return out.ravel()


def simulate(mesh, beta0, *, pump, time, sigma_ase, phi_history=None, phi_prism_history=None):
    """beta after every step ([steps + 1][P]) and the absorbed pump fraction per step.
    phi_history: per-sample phi of every ASE solve, in order (a prism's phi is
    the mean of its six vertices); phi_prism_history: per-prism phi of every
    ASE solve (the forward method's volume-weighted cell means) used as given."""
    sA, sE = sigma_ase
    P = mesh.numberOfPrisms
    clad = np.zeros(P, bool)
    if mesh.claddingCellTypes is not None:
        clad = np.tile(mesh.claddingCellTypes == mesh.claddingNumber, mesh.numberOfLevels - 1)
    beta = np.asarray(beta0, np.float64).copy()
    hist = [beta.copy()]
    absorbed = []
    dt, tau = time["timeStep"], mesh.crystalTFluo
    method = int(time.get("integrator", 0))
    iterations = max(1, int(time.get("implicitIterations", 0)) or 8)
    solve = 0  # phi-ASE solves consumed so far

    def next_phi():
        nonlocal solve
        if phi_prism_history is not None:
            v = np.asarray(phi_prism_history[solve], np.float32).astype(np.float64)
        else:
            v = prism_phi(mesh, phi_history[solve]).astype(np.float64)
        solve += 1
        return v

    for step in range(time["steps"]):
        ase = step < time["aseSteps"]
        pump_on = step < time["pumpSteps"]
        state = {"phi": np.zeros(P), "first_pump": True}

        def pump_at(b):
            if not pump_on:
                return np.zeros(P)
            rate, absd, inc = pump_rate(mesh, b, pump, clad)
            if state["first_pump"]:
                absorbed.append(absd / inc if inc > 0 else 0.0)
            state["first_pump"] = False
            return rate

        def deriv(b, refresh=True):
            if ase and refresh:
                state["phi"] = next_phi()
            k = pump_at(b) - (b * (sE + sA) - sA) * state["phi"] - b / tau
            return np.where(clad, 0.0, k)

        if not pump_on:
            absorbed.append(0.0)
        if method in (0, 4):  # RK4; 0: phi-ASE frozen at the step start
            k1 = deriv(beta)
            k2 = deriv(beta + 0.5 * dt * k1, method == 4)
            k3 = deriv(beta + 0.5 * dt * k2, method == 4)
            k4 = deriv(beta + dt * k3, method == 4)
            new = beta + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
        elif method == 2:  # heun
            k1 = deriv(beta)
            k2 = deriv(beta + dt * k1)
            new = beta + 0.5 * dt * (k1 + k2)
        elif method == 3:  # midpoint
            k1 = deriv(beta)
            new = beta + dt * deriv(beta + 0.5 * dt * k1)
        elif method == 5:  # implicit euler: stage = beta + dt k(stage), fixed-point iterations
            stage = beta
            for _ in range(iterations):
                stage = beta + dt * deriv(stage)
            new = stage
        elif method == 6:  # exponential euler
            if ase:
                state["phi"] = next_phi()
            rate = pump_at(beta)
            decay = np.exp(-dt / tau)
            source = np.where(clad, 0.0, rate - (beta * (sE + sA) - sA) * state["phi"])
            new = tau * source * (1.0 - decay) + beta * decay
        else:  # explicit euler
            new = beta + dt * deriv(beta)
        # clipped to [0, 1] after every update (include/kernels/timeIntegrationUpdateKernels.hpp:93-105)
        beta = np.clip(new, 0.0, 1.0)
        hist.append(beta.copy())
    return np.array(hist), np.array(absorbed)
