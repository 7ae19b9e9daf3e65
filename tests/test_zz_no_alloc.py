"""The allocation-free entry point, sbe_solve_noalloc.

It exists for callers that must not allocate device memory themselves (code
inside an application whose device memory belongs to that application's pool
allocator, or latency-critical loops where cudaMalloc/cudaFree could
synchronise the device): all of its working memory is one fixed array inside
the library.  Here it is called through the C ABI twice in a row per problem
(the second call reuses the array the first one left behind) and compared
with the regular entry point (sbe_solver_create/run/get) at the tolerance of
the GPU parity tests.  This file sorts last so that a run stopping at the
first failure has already run every other test."""
import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200.api import SbeError, solve_noalloc
from cases import GOLDEN_CASES, variant

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-10


def _rel(a, b, scale):
    m = max(np.abs(b).max(), 1e-5 * scale)
    return np.abs(a - b).max() / m


def _check(out, ref):
    scale = max(np.abs(ref.inter).max(), np.abs(ref.intra).max())
    for key in ("inter", "intra"):
        for a in range(3):
            assert _rel(getattr(out, key)[:, a], getattr(ref, key)[:, a], scale) < FP64_TOL, (key, a)
    assert np.abs(out.occ - ref.occ).max() < 1e-12
    assert np.abs(out.coh - ref.coh).max() < 1e-12
    assert np.array_equal(out.laser, ref.laser)


@pytest.mark.parametrize("case,opts", [
    (GOLDEN_CASES["vg_rk4"], dict(precision="fp64")),
    (GOLDEN_CASES["lw_t1_elliptic"], dict(precision="fp64")),
    (variant(calc__Npoints=[40, 33], calc__RKorder=5), dict(precision="fp64", tile_k=256, k_per_thread=2)),
])
def test_noalloc_matches_regular_entry_point_twice(case, opts):
    p = ab.Problem.from_dict(case)
    ref = ab.solve(p, **opts)
    first = solve_noalloc(p, **opts)
    second = solve_noalloc(p, **opts)
    _check(first, ref)
    _check(second, ref)


@pytest.mark.parametrize("kpt", [1, 2])
def test_noalloc_mixed_precision_twice(kpt):
    p = ab.Problem.from_dict(variant(calc__Npoints=[24, 24]))
    opts = dict(precision="mixed", tile_k=64 * kpt, k_per_thread=kpt)   # same launch shape on both paths
    ref = ab.solve(p, **opts)
    for _ in range(2):
        out = solve_noalloc(p, **opts)
        # same kernels and tiling: the mixed results agree to FP64 rounding of the k-sum
        _check(out, ref)


def test_noalloc_rejects_problems_beyond_its_scratch():
    big = ab.Problem.from_dict(variant(calc__Npoints=[700, 700]))
    with pytest.raises(SbeError) as e:
        solve_noalloc(big, precision="fp64")
    assert e.value.name == "SBE_OOM" and "bytes of device scratch" in str(e.value)
