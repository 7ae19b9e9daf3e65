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
    # length gauge, Fehlberg-5: six stage-time columns of the field table
    (variant(top__gauge="Wannier", calc__Npoints=[21, 17], calc__RKorder=5), dict(precision="fp64", tile_k=64)),
    # length gauge, mixed: the twelve cos/sin columns rounded to float
    (variant(top__gauge="Wannier", calc__Npoints=[21, 17]), dict(precision="mixed", tile_k=64)),
    (variant(top__gauge="Wannier", calc__Npoints=[19, 15], calc__RKorder=5, calc__T1=300.0),
     dict(precision="mixed", tile_k=96, k_per_thread=1)),
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


@pytest.mark.parametrize("gauge", ["Velocity", "Wannier"])
def test_noalloc_default_options_match_regular_defaults(gauge):
    """With no launch options both entry points pick their own shapes (the
    regular one may autotune); FP64 results differ only in the k-sum's order."""
    p = ab.Problem.from_dict(variant(top__gauge=gauge, calc__Npoints=[33, 29]))
    ref = ab.solve(p, precision="fp64")
    for _ in range(2):
        _check(solve_noalloc(p, precision="fp64"), ref)


def test_noalloc_default_mixed_matches_regular_default():
    """Mixed velocity gauge with default options: both paths use the packed
    two-k-point kernel; the FP32 warp sums group k-points by tile, so the
    agreement is to FP32 rounding of the k-sum."""
    p = ab.Problem.from_dict(variant(calc__Npoints=[33, 29]))
    ref = ab.solve(p, precision="mixed")
    out = solve_noalloc(p, precision="mixed")
    scale = max(np.abs(ref.inter).max(), np.abs(ref.intra).max())
    for key in ("inter", "intra"):
        assert np.abs(getattr(out, key) - getattr(ref, key)).max() < 1e-5 * scale, key


def test_noalloc_rejects_bad_launch_shapes_before_any_work():
    p = ab.Problem.from_dict(variant())
    for opts in (dict(tile_k=192, k_per_thread=3), dict(tile_k=48), dict(tile_k=1024)):
        with pytest.raises(SbeError) as e:
            solve_noalloc(p, precision="fp64", **opts)
        assert e.value.name == "SBE_INVALID_ARGUMENT", opts
    # the entry point still works after the rejections
    _check(solve_noalloc(p, precision="fp64"), ab.solve(p, precision="fp64"))
