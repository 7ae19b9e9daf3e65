"""The CPU oracle (oracle/sbe_oracle.c) against outputs of the reference
itself (golden fixtures made by tests/golden/make_golden.py from the
unmodified reference sources).  This pins the oracle before the GPU kernels are
compared with it."""
import copy
import os

import numpy as np
import pytest

from cases import BAND_GROUPS, GOLDEN_CASES, MATERIAL_CASES, MULTIWSM_CASES, SNAPSHOT_CASES
from oracle import pyoracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    m = np.abs(b).max()
    return np.abs(a - b).max() / (m if m > 0 else 1.0)


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES) + sorted(MULTIWSM_CASES))
def test_oracle_matches_reference_outputs(name):
    case = {**GOLDEN_CASES, **MULTIWSM_CASES}[name]
    ref = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    out = pyoracle.run(case)
    N = out["dims"]["nband"]
    # the files hold 17 significant digits; the oracle repeats the
    # reference's arithmetic, so the match is to the last printed digit
    assert _rel(out["inter"], ref["inter"]) < 1e-15
    assert _rel(out["intra"], ref["intra"]) < 1e-15
    occ = ref["occ_file"]
    assert np.abs(out["occ"] - occ[:, :N]).max() < 1e-15
    assert np.abs(out["occ"].sum(1) - occ[:, N]).max() < 1e-14
    # laser file: time axis and the A/E columns
    t = out["dims"]["atmin"] + case["calc"].get("dt", 0.1) * np.arange(out["dims"]["Nt"])
    assert np.allclose(ref["laser"][:, 0], t, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("name", sorted(MATERIAL_CASES))
def test_material_tables_reproduce_reference_outputs(name):
    """The analytic materials as Fourier tables (read from the product's cfg
    front end) run through the oracle's engine against the reference's own
    run of the same cfg: the tables reproduce each material's H and GenJMatrix
    and the engine its propagation, to summation-order rounding."""
    case = MATERIAL_CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    out = pyoracle.run(case)
    N = out["dims"]["nband"]
    assert _rel(out["inter"], ref["inter"]) < 1e-12
    assert _rel(out["intra"], ref["intra"]) < 1e-12
    for g in BAND_GROUPS.get(name, [[n] for n in range(N)]):
        assert np.abs(out["occ"][:, g].sum(1) - ref["occ_file"][:, g].sum(1)).max() < 1e-13, g


def test_oracle_threads_match_sequential():
    """The ParaRange k-split (utility.h:104-115) changes only summation order."""
    case = GOLDEN_CASES["vg_rk4"]
    a = pyoracle.run(case, nthreads=1)
    b = pyoracle.run(case, nthreads=3)
    assert _rel(b["inter"], a["inter"]) < 1e-13
    assert _rel(b["intra"], a["intra"]) < 1e-13


def test_oracle_eigh_against_numpy():
    rng = np.random.default_rng(7)
    for n in (2, 3, 6, 8):
        a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        a = a + a.conj().T
        w, v = pyoracle.eigh(a)
        assert np.allclose(w, np.linalg.eigvalsh(a), atol=1e-12)
        assert np.allclose(a @ v, v * w, atol=1e-11)
        assert np.allclose(v.conj().T @ v, np.eye(n), atol=1e-12)


def test_oracle_haldane_j_is_minus_dh_dk():
    case = GOLDEN_CASES["vg_rk4"]
    k = np.array([0.31, -0.17, 0.0])
    _, J = pyoracle.model_hj(case, k)
    h = 1e-6
    for a in range(2):
        dk = np.zeros(3)
        dk[a] = h
        Hp, _ = pyoracle.model_hj(case, k + dk)
        Hm, _ = pyoracle.model_hj(case, k - dk)
        assert np.allclose(J[a], -(Hp - Hm) / (2 * h), atol=1e-8)
    assert np.all(J[2] == 0)


@pytest.mark.parametrize("n", [1.0, 2.0, 1.5])
def test_oracle_multiwsm_j_is_minus_dh_dk(n):
    """MultiWSM's GenJMatrix formulas (MultiWSM.h:84-147) are -dH/dk of its
    GenBcomp (MultiWSM.h:186-200) away from the k_x = k_y = 0 line, z included."""
    case = copy.deepcopy(MULTIWSM_CASES["multiwsm_w"])
    case["MultiWSM"]["n"] = n
    k = np.array([0.31, -0.17, 0.4])
    _, J = pyoracle.model_hj(case, k)
    h = 1e-6
    for a in range(3):
        dk = np.zeros(3)
        dk[a] = h
        Hp, _ = pyoracle.model_hj(case, k + dk)
        Hm, _ = pyoracle.model_hj(case, k - dk)
        assert np.allclose(J[a], -(Hp - Hm) / (2 * h), atol=1e-8), a
    assert np.allclose(J[2], np.diag([-0.2, 0.2]))


def test_multiwsm_problem_matches_oracle_grid():
    """The cfg front end's MultiWSM problem: the oracle's 3-D grid and zone
    (the cube [-pi/a0, pi/a0]^3, a0 in Angstrom)."""
    from antelope_b200 import Problem

    for name, case in MULTIWSM_CASES.items():
        d, od = Problem.from_dict(case).dims, pyoracle.dims(case)
        assert (d.ntotal, d.Nt, d.nband, d.nval) == (od["ntotal"], od["Nt"], od["nband"], od["nval"]), name
        assert d.dV == od["dV"], name


@pytest.mark.skipif(not os.path.exists(pyoracle.REF_EXE), reason="reference build absent")
def test_oracle_matches_live_reference_build(tmp_path):
    """Re-run one case through the reference build when it is present."""
    case = GOLDEN_CASES["lw_t1_elliptic"]
    ref = pyoracle.run_reference(case, str(tmp_path))
    out = pyoracle.run(case)
    assert _rel(out["inter"], ref["inter"]) < 1e-15
    assert _rel(out["intra"], ref["intra"]) < 1e-15


@pytest.mark.parametrize("name", sorted(SNAPSHOT_CASES))
def test_oracle_snapshots_match_reference(name):
    """Density snapshots (calc.shotNumber, antelope.cpp:267-422) against the
    reference's snapshot files.  occupation_1d_integration.dat is printed with
    %16e (7 significant digits).  The reference's binary files index the k
    loop with a stale k index (antelope.cpp:384-400): in the velocity gauge
    every entry holds the last k-point's value, in the length gauge only the
    last entry is set; the oracle stores each k's own value, so the last entry
    is compared (the coherence by modulus: it carries the eigenvector phases)."""
    case = SNAPSHOT_CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    out = pyoracle.run(case)
    _, ns = pyoracle.shot_dims(case)
    nt = out["dims"]["ntotal"]
    assert ref["occ1d"].shape == out["occ1d"].shape == (ns, case["calc"]["Npoints"][0])
    # (values at rounding-noise level, ~1e-17 right after the first step, get
    # an absolute floor of 1e-13 of the largest value)
    floor = 1e-13 * np.abs(ref["occ1d"]).max()
    assert np.all(np.abs(out["occ1d"] - ref["occ1d"]) <= 6e-7 * np.abs(ref["occ1d"]) + floor)
    rn, rp = ref["nc"].reshape(ns, nt), ref["pi"].reshape(ns, nt)
    assert np.abs(out["nc"][:, -1] - rn[:, -1]).max() < 1e-13
    assert np.abs(np.abs(out["pi"][:, -1]) - np.abs(rp[:, -1])).max() < 1e-13
    if case.get("gauge") == "Velocity":
        assert np.array_equal(rn, np.repeat(rn[:, -1:], nt, axis=1))   # the reference's stale index
    # the 1-D integration is the weighted sum of the per-k values
    k, w = pyoracle.kgrid(case)
    n0, n1 = case["calc"]["Npoints"][0], case["calc"]["Npoints"][1]
    s = (out["nc"] * w).reshape(ns, n0, -1).sum(2) / n1
    assert np.abs(s - out["occ1d"]).max() < 1e-15


def test_oracle_snapshot_threads_match_sequential():
    case = SNAPSHOT_CASES["lw_shots"]
    a = pyoracle.run(case, nthreads=1)
    b = pyoracle.run(case, nthreads=3)
    assert np.array_equal(a["nc"], b["nc"]) and np.array_equal(a["pi"], b["pi"])
    assert np.abs(a["occ1d"] - b["occ1d"]).max() < 1e-16
