"""Synthetic inputs of the benchmark shapes (no public dataset is involved).

haldane_case  -- the two-band Haldane problem of the plain-method and
                 600x600 configurations: a0 = 1.44 A, t1 = 0.075, t2 = t1/3,
                 phi0 = 1.16, M = 2.54 t2; 3.2 um (w0 = 0.014238 a.u.),
                 E0 = 0.0045 a.u., 8-cycle sin^2 envelope; velocity gauge,
                 dt = 0.1 a.u. (~35.3k steps), RK4, T2 = 220 a.u.
scan_cases    -- the seeded 256-solve parameter scan (uneven grids 100^2..400^2,
                 4..12 cycles, M/t2 in [-4,4], phi0 in [0,pi], ellipticity in
                 {0,.25,.5,1} x helicity, CEP in [0,360) deg).
serving_cases -- the seeded Poisson request stream (Haldane and two-colour
                 w + 2w requests, 64^2..512^2, 4..16 cycles, 1.6..3.2 um,
                 E0 in [0.002, 0.006]).
"""
from __future__ import annotations

import copy

import numpy as np

AU_LIGHT = 137.035999
BOHR_NM = 0.0529177210903


def omega_of_um(lam_um: float) -> float:
    """Photon energy (a.u.) of a wavelength in micrometres."""
    return 2 * np.pi * AU_LIGHT / (lam_um * 1000.0 / BOHR_NM)


def haldane_case(n: int = 150, precision: str = "fp64", env: str = "sin2", ncycles: float = 8.0,
                 gauge: str = "Velocity") -> dict:
    return {
        "target": "Haldane",
        "gauge": gauge,
        "laser": {"offset": [0.0, 0.0],
                  "pulses": [{"E0": 0.0045, "w0": 0.014238, "ncycles": float(ncycles), "ellip": 0.0,
                              "cep": 0.0, "t0": 0.0, "phix": 0.0, "env_name": env}]},
        "calc": {"Npoints": [n, n], "dt": 0.1, "T1": -1.0, "T2": 220.0, "RKorder": 4, "InterIntra": True,
                 "ksfactor": [1.0, 1.0, 1.0], "precision": precision},
        "Haldane": {"a0": 1.44, "t1": 0.075, "t2": 0.025, "Mt2": 2.54, "phi0": 1.16},
    }


def scan_cases(n: int = 256, seed: int = 20261203, precision: str = "mixed", grid_scale: float = 1.0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        c = haldane_case(precision=precision)
        g = int(rng.choice([100, 200, 300, 400]) * grid_scale)
        c["calc"]["Npoints"] = [max(g, 4), max(g, 4)]
        p = c["laser"]["pulses"][0]
        p["ncycles"] = float(rng.integers(4, 13))
        p["ellip"] = float(rng.choice([0.0, 0.25, 0.5, 1.0]) * rng.choice([-1.0, 1.0]))
        p["cep"] = float(rng.uniform(0.0, 360.0))
        c["Haldane"]["Mt2"] = float(rng.uniform(-4.0, 4.0))
        c["Haldane"]["phi0"] = float(rng.uniform(0.0, np.pi))
        out.append(c)
    return out


def serving_cases(n: int = 2000, seed: int = 20261204, rate_hz: float = 20.0, precision: str = "mixed",
                  grid_scale: float = 1.0):
    """Returns (arrival_times_s, cases)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=n))
    out = []
    for _ in range(n):
        c = haldane_case(precision=precision)
        g = int(rng.integers(64, 513) * grid_scale)
        c["calc"]["Npoints"] = [max(g, 4), max(g, 4)]
        lam = float(rng.uniform(1.6, 3.2))
        w0 = omega_of_um(lam)
        p = c["laser"]["pulses"][0]
        p["w0"] = w0
        p["E0"] = float(rng.uniform(0.002, 0.006))
        p["ncycles"] = float(rng.integers(4, 17))
        if rng.random() < 0.5:  # two-colour w + 2w with the same envelope duration
            q = copy.deepcopy(p)
            q["w0"] = 2 * w0
            q["E0"] = p["E0"] * float(rng.uniform(0.1, 0.5))
            q["ncycles"] = 2 * p["ncycles"]
            q["cep"] = float(rng.uniform(0.0, 360.0))
            c["laser"]["pulses"].append(q)
        out.append(c)
    return t, out
