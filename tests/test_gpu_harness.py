"""The GPU kernels against the harness build of the reference (the reference's
own SBEs/laser code with the sin2 envelope and the SyntheticWannier material
with dipole matrices, oracle/make_harness.py; golden fixtures made by
tests/golden/make_golden.py): the headline sin2 pulse on the closed-form
Haldane kernels, and the N-band kernels with the length gauge's E(t).D(k+A)
term (SBEs.h:771-782) and the current operator -dH/dk + i[D, H]
(BaseMaterial.h:62-68).  FP64 bar: 1e-10 of max_t |J| per current series,
occupations 1e-12.  The adaptive Cash-Karp extension is checked against the
reference's fine fixed-step solution of the same equations."""
import copy
import os

import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200.api import Solver
from cases import HARNESS_CASES

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-10


def rel_series(a, b, scale):
    # a series that vanishes by symmetry up to rounding noise is measured
    # against 1e-5 of the run's largest current
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-5 * scale)


@pytest.mark.parametrize("name", sorted(n for n in HARNESS_CASES if not n.endswith("_fine")))
def test_fp64_matches_harness_reference(name):
    case = HARNESS_CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    out = ab.solve(case, precision="fp64")
    scale = max(np.abs(ref["inter"]).max(), np.abs(ref["intra"]).max())
    for key in ("inter", "intra"):
        for a in range(3):
            assert rel_series(getattr(out, key)[:, a], ref[key][:, a], scale) < FP64_TOL, (key, a)
    assert np.abs(out.occ - ref["occ_file"]).max() < 1e-12


def test_cashkarp_converges_to_the_reference_fine_solution():
    """Cash-Karp on the GPU with an output interval of 0.5 and tolerance 1e-12
    (the controller cuts the step) against the reference's own Fehlberg-5 at
    dt = 0.025 on the same N = 6 model with dipoles."""
    fine = np.load(os.path.join(GOLDEN, "golden_synw6_w_rk5_fine.npz"))
    c = copy.deepcopy(HARNESS_CASES["synw6_w_rk4"])
    c["calc"].update(rk="cashkarp45", dt=0.5, tol=1e-12)
    s = Solver(ab.Problem.from_dict(c), precision="fp64")
    s.run()
    out = s.get()
    st = s.steps()
    s.close()
    n = out.inter.shape[0]
    ref = fine["inter"][::20][:n]
    assert st["steps"] > 2 * n
    assert np.abs(out.inter - ref).max() / np.abs(ref).max() < 2e-10
