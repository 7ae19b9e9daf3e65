"""k-sharding of one solve (the reference's ParaRange split of the k-grid over
MPI ranks and the final MPI_Reduce, antelope.cpp:152, 482-512): solves of
k-slices run one after another on one GPU, their k-sums added and assembled,
against the whole solve.  Tiles differ between the slices and the whole grid,
so sums are grouped differently: agreement to rounding (1e-12 of max |J|)."""
import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200.api import Solver, assemble
from antelope_b200.dist import para_range
from cases import GOLDEN_CASES, MATERIAL_CASES

pytestmark = pytest.mark.gpu


def sharded(problem, n, precision):
    total = None
    for r in range(n):
        s = Solver(problem, k_slice=para_range(problem.dims.ntotal, n, r), precision=precision)
        s.run()
        part = s.sums()
        s.close()
        total = part if total is None else total + part
    return assemble(problem, total)


@pytest.mark.parametrize("name,n", [("vg_rk4", 3), ("lw_rk4", 2), ("vg_fermi_t1", 4), ("kanemele_w", 3),
                                    ("haldane2l_v", 2)])
def test_slices_add_up_to_the_whole_solve(name, n):
    case = GOLDEN_CASES.get(name) or MATERIAL_CASES[name]
    p = ab.Problem.from_dict(case)
    full = ab.solve(case, precision="fp64")
    got = sharded(p, n, "fp64")
    scale = max(np.abs(full.inter).max(), np.abs(full.intra).max())
    for key in ("inter", "intra"):
        assert np.abs(getattr(got, key) - getattr(full, key)).max() < 1e-12 * scale, key
    assert np.abs(got.occ - full.occ).max() < 1e-13
    assert np.array_equal(got.laser, full.laser)


def test_assemble_of_whole_sums_is_get():
    case = GOLDEN_CASES["vg_rk4"]
    p = ab.Problem.from_dict(case)
    s = Solver(p, precision="fp64")
    s.run()
    a = s.get()
    b = assemble(p, s.sums())
    s.close()
    for key in ("inter", "intra", "occ", "coh", "laser"):
        assert np.array_equal(getattr(a, key), getattr(b, key)), key


def test_bad_slice_is_rejected():
    p = ab.Problem.from_dict(GOLDEN_CASES["vg_rk4"])
    with pytest.raises(ab.SbeError):
        Solver(p, k_slice=(5, 5))
