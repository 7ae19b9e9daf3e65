"""Harmonic band powers computed on the GPU from the device-resident results
(sbe_solver_harmonics / sbe_batch_harmonics) against the same convention
applied with numpy's FFT to the solve's written outputs
(antelope_b200/spectrum.py, AnalysisReader_PyDir.py:252-354).  The direct
DFT and the FFT differ by rounding only: bands down to 1e-8 of the strongest
agree to 1e-7 relative."""
import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200 import wannier
from antelope_b200.spectrum import harmonic_powers, spectrum
from cases import GOLDEN_CASES, MATERIAL_CASES

pytestmark = pytest.mark.gpu


def reference_bands(out, dt, w0, hmax):
    w, S = spectrum(out.inter, out.intra, dt)
    return harmonic_powers(w, S, w0, hmax)


def check(bands, ref):
    keep = ref >= 1e-8 * ref.max()
    assert keep.sum() >= 3
    rel = np.abs(bands[keep] - ref[keep]) / ref[keep]
    assert rel.max() < 1e-7, rel


@pytest.mark.parametrize("name,prec", [("vg_rk4", "fp64"), ("lw_rk4", "fp64"), ("vg_two_color", "mixed"),
                                       ("vg_total_current", "fp64")])
def test_haldane_harmonics(name, prec):
    case = GOLDEN_CASES[name]
    w0, hmax = case["laser"]["pulses"][0]["w0"], 12
    s = ab.api.Solver(ab.Problem.from_dict(case), precision=prec)
    s.run()
    out = s.get()
    bands = s.harmonics(w0, hmax)
    s.close()
    check(bands, reference_bands(out, case["calc"]["dt"], w0, hmax))


@pytest.mark.parametrize("name", ["kanemele_w", "haldane2l_v"])
def test_table_model_harmonics(name):
    case = MATERIAL_CASES[name]
    w0, hmax = case["laser"]["pulses"][0]["w0"], 10
    s = ab.api.Solver(ab.Problem.from_dict(case), precision="fp64")
    s.run()
    out = s.get()
    bands = s.harmonics(w0, hmax)
    s.close()
    check(bands, reference_bands(out, case["calc"]["dt"], w0, hmax))


def test_batch_harmonics():
    cases = [GOLDEN_CASES["vg_rk4"], GOLDEN_CASES["vg_fermi_t1"]]
    probs = [ab.Problem.from_dict(c) for c in cases]
    b = ab.Batch(probs, precision="fp64")
    b.run()
    for i, c in enumerate(cases):
        w0 = c["laser"]["pulses"][0]["w0"]
        check(b.harmonics(i, w0, 10), reference_bands(b.get(i), c["calc"]["dt"], w0, 10))
    b.close()
