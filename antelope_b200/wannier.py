"""Synthetic Wannier tight-binding models (the N-band model form of
src/GeneralModel/Materials/Wannier90.h:297-387, without a Wannier90 file).

H(k) = sum_R h_R e^{i k.R},  D_a(k) = sum_R d_{a,R} e^{i k.R}  (a = x, y),
R = n1 a1 + n2 a2 on a 2-D lattice, h_{-R} = h_R^dagger and
d_{a,-R} = d_{a,R}^dagger so H and D are Hermitian.

A model travels inside inputParam.cfg as explicit arrays of the
``SyntheticWannier`` group, so every consumer (the GPU library, the CPU
oracle, the tests) reads the identical numbers:

    SyntheticWannier = {
        Nband = 6; Nval = 3;
        lattice = [a1x, a1y, a2x, a2y];      # bohr
        R = [n1, n2, n1, n2, ...];           # integer lattice coordinates
        h_re = [...]; h_im = [...];          # [nR][N][N], a.u.
        d_re = [...]; d_im = [...];          # [nR][2][N][N], bohr (optional)
    };

``generate`` draws the seeded model of the N = 6 benchmark configuration:
triangular lattice a = 2.72 bohr, the 37 vectors with |R| <= 3a, complex
Gaussian hoppings with variance decaying as exp(-|R|/a), dipoles from the
same distribution scaled by 0.5, and an on-site splitting that puts the Nval
lowest bands below the others.
"""
from __future__ import annotations

import numpy as np


def lattice_vectors(a: float = 2.72):
    return np.array([[a, 0.0], [0.5 * a, 0.5 * np.sqrt(3.0) * a]])


def shell_vectors(a: float = 2.72, rmax: float = 3.0):
    """Integer coordinates (n1, n2) of all R with |R| <= rmax * a, sorted by
    length then angle (37 vectors for rmax = 3 on the triangular lattice)."""
    L = lattice_vectors(a)
    out = []
    m = int(np.ceil(rmax)) + 2
    for n1 in range(-m, m + 1):
        for n2 in range(-m, m + 1):
            r = n1 * L[0] + n2 * L[1]
            if np.linalg.norm(r) <= rmax * a * (1 + 1e-12):
                out.append((n1, n2, np.linalg.norm(r), np.arctan2(r[1], r[0])))
    out.sort(key=lambda x: (round(x[2], 9), x[3]))
    return np.array([(o[0], o[1]) for o in out], dtype=np.int32)


def generate(seed: int, nband: int = 6, nval: int = 3, a: float = 2.72, rmax: float = 3.0,
             h_scale: float = 0.02, d_ratio: float = 0.5, gap: float = 0.2) -> dict:
    """The cfg group (dict) of a seeded synthetic model."""
    rng = np.random.default_rng(seed)
    R = shell_vectors(a, rmax)
    L = lattice_vectors(a)
    nR, N = len(R), nband
    idx = {tuple(r): i for i, r in enumerate(R)}
    h = np.zeros((nR, N, N), dtype=np.complex128)
    d = np.zeros((nR, 2, N, N), dtype=np.complex128)

    def cg(shape, std):
        return std * (rng.normal(size=shape) + 1j * rng.normal(size=shape)) / np.sqrt(2.0)

    for i, r in enumerate(R):
        j = idx[(-r[0], -r[1])]
        if j < i:
            continue
        std = h_scale * np.exp(-0.5 * np.linalg.norm(r[0] * L[0] + r[1] * L[1]) / a)
        hm = cg((N, N), std)
        dm = cg((2, N, N), d_ratio * std / h_scale)
        if i == j:  # R = 0: Hermitian on-site block
            hm = 0.5 * (hm + hm.conj().T)
            dm = 0.5 * (dm + np.conj(np.swapaxes(dm, 1, 2)))
            hm += np.diag([-0.5 * gap] * nval + [0.5 * gap] * (N - nval))
            h[i], d[i] = hm, dm
        else:
            h[i], h[j] = hm, hm.conj().T
            d[i], d[j] = dm, np.conj(np.swapaxes(dm, 1, 2))
    return {"Nband": N, "Nval": nval, "lattice": [float(x) for x in L.reshape(-1)],
            "R": [int(x) for x in R.reshape(-1)],
            "h_re": [float(x) for x in h.real.reshape(-1)], "h_im": [float(x) for x in h.imag.reshape(-1)],
            "d_re": [float(x) for x in d.real.reshape(-1)], "d_im": [float(x) for x in d.imag.reshape(-1)]}


def synthetic_model(group: dict) -> dict:
    """Arrays of a model from its cfg group (inverse of ``generate``)."""
    N = int(group["Nband"])
    R = np.asarray(group["R"], dtype=np.int32).reshape(-1, 2)
    nR = len(R)
    h = (np.asarray(group["h_re"]) + 1j * np.asarray(group["h_im"])).reshape(nR, N, N)
    d = None
    if "d_re" in group:
        d = (np.asarray(group["d_re"]) + 1j * np.asarray(group["d_im"])).reshape(nR, 2, N, N)
    return {"nband": N, "nval": int(group["Nval"]), "R": R, "h": h, "d": d,
            "lattice": [float(x) for x in group["lattice"]]}


def wannier_case(seed: int, n: int = 300, precision: str = "fp64", ncycles: float = 10.0,
                 rk: str = "cashkarp45", tol: float = 1e-8, gauge: str = "Wannier") -> dict:
    """The N = 6 benchmark problem: 3.2 um pulse, T2 = 220, Cash-Karp RK45."""
    calc = {"Npoints": [n, n], "dt": 0.1, "T1": -1.0, "T2": 220.0, "RKorder": 4, "InterIntra": True,
            "ksfactor": [1.0, 1.0, 1.0], "precision": precision}
    if rk:
        calc["rk"] = rk
        calc["tol"] = tol
    return {"target": "SyntheticWannier", "gauge": gauge,
            "laser": {"offset": [0.0, 0.0],
                      "pulses": [{"E0": 0.0045, "w0": 0.014238, "ncycles": float(ncycles), "ellip": 0.0,
                                  "cep": 0.0, "t0": 0.0, "phix": 0.0, "env_name": "sin2"}]},
            "calc": calc, "SyntheticWannier": generate(seed)}
