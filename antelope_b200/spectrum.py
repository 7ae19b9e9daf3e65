"""HHG spectrum and the per-harmonic error used to qualify the mixed-precision
method.

Spectrum convention of the reference's analysis script
(src/GeneralModel/AlsisPythonShort/AnalysisReader_PyDir.py:252-354): Blackman
window over the whole record, FFT times dt, multiplied by -i*omega after
fftshift (that is FFT of dJ/dt), |.|^2 summed over x and y, with
J = interband + intraband current per axis.  Harmonic bands are the order
ranges h +/- 1/2 (as in IntegrateSpectrumOrder.py:57-70).
"""
from __future__ import annotations

import numpy as np


def spectrum(inter: np.ndarray, intra: np.ndarray, dt: float):
    """Return (omega, S) with S(omega) = sum_{x,y} |-i omega FFT(w J) dt|^2."""
    J = np.asarray(inter, dtype=np.float64)[:, :2] + np.asarray(intra, dtype=np.float64)[:, :2]
    Nt = J.shape[0]
    win = np.blackman(Nt)
    w = 2 * np.pi * np.fft.fftshift(np.fft.fftfreq(Nt, dt))
    S = np.zeros(Nt)
    for a in range(2):
        F = np.fft.fftshift(np.fft.fft(win * J[:, a]) * dt)
        S += np.abs(-1j * w * F) ** 2
    return w, S


def harmonic_powers(omega: np.ndarray, S: np.ndarray, w0: float, hmax: int | None = None):
    """Band power of harmonic orders h = 1..hmax (sum of S over |w/w0 - h| < 1/2)."""
    order = omega / w0
    if hmax is None:
        hmax = int(np.floor(order.max() - 0.5))
    out = np.zeros(hmax)
    for h in range(1, hmax + 1):
        m = (order >= h - 0.5) & (order < h + 0.5)
        out[h - 1] = S[m].sum()
    return out


def per_harmonic_error(test: dict, ref: dict, dt: float, w0: float, floor: float = 1e-8,
                       hmax: int | None = None):
    """Relative error of each harmonic band's power, over the harmonics whose
    reference band power is at least ``floor`` times the strongest one.
    ``test``/``ref`` hold 'inter' and 'intra' arrays [Nt, 3].  Returns
    (orders, errors, reference band powers)."""
    w, St = spectrum(test["inter"], test["intra"], dt)
    _, Sr = spectrum(ref["inter"], ref["intra"], dt)
    Pt = harmonic_powers(w, St, w0, hmax)
    Pr = harmonic_powers(w, Sr, w0, hmax)
    keep = Pr >= floor * Pr.max()
    orders = np.nonzero(keep)[0] + 1
    err = np.abs(Pt[keep] - Pr[keep]) / Pr[keep]
    return orders, err, Pr[keep]
