"""The CPU oracle (oracle/sbe_oracle.c) against outputs of the reference
itself (golden fixtures made by tests/golden/make_golden.py from the
unmodified reference sources).  This pins the oracle before the GPU kernels are
compared with it."""
import copy
import os

import numpy as np
import pytest

from cases import BAND_GROUPS, GOLDEN_CASES, HARNESS_CASES, MATERIAL_CASES, MULTIWSM_CASES, SNAPSHOT_CASES
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


HARNESS_PINNED = sorted(n for n in HARNESS_CASES if not n.endswith("_fine"))


@pytest.mark.parametrize("name", HARNESS_PINNED)
def test_oracle_matches_harness_reference(name):
    """The sin2 envelope and the N-band SyntheticWannier model with dipole
    matrices, run by the reference's own SBEs/laser code (the harness build
    of oracle/make_harness.py): the oracle repeats its arithmetic to the last
    printed digit -- the E(t).D(k+A) term of the length gauge (SBEs.h:771-782),
    the current operator -dH/dk + i[D, H] (BaseMaterial.h:62-68) in both
    gauges, RK4 and Fehlberg-5, T1 and elliptic pulses."""
    case = HARNESS_CASES[name]
    ref = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    out = pyoracle.run(case)
    N = out["dims"]["nband"]
    assert _rel(out["inter"], ref["inter"]) < 1e-15
    assert _rel(out["intra"], ref["intra"]) < 1e-15
    assert np.abs(out["occ"] - ref["occ_file"][:, :N]).max() < 1e-15
    assert np.abs(out["occ"].sum(1) - ref["occ_file"][:, N]).max() < 1e-14


def test_harness_dipoles_enter_the_length_gauge():
    """The dipole matrices change the reference's length-gauge currents well
    beyond rounding, so the pinned cases exercise the E.D and i[D, H] terms."""
    a = np.load(os.path.join(GOLDEN, "golden_synw6_w_rk4.npz"))
    b = np.load(os.path.join(GOLDEN, "golden_synw6_w_rk4_no_dipoles.npz"))
    assert _rel(b["inter"], a["inter"]) > 1e-2
    assert _rel(b["intra"], a["intra"]) > 1e-3


def _order_conditions(c, a, b):
    """Residuals of the Runge-Kutta order conditions (the rooted trees up to
    order 5, Butcher) for weights b: order p holds when the residuals of all
    trees with at most p nodes vanish.  Returns {order: max residual}."""
    ac = a @ c
    acc = a @ (c * c)
    aac = a @ ac
    conds = {
        1: [b.sum() - 1],
        2: [b @ c - 1 / 2],
        3: [b @ (c * c) - 1 / 3, b @ ac - 1 / 6],
        4: [b @ c ** 3 - 1 / 4, b @ (c * ac) - 1 / 8, b @ acc - 1 / 12, b @ aac - 1 / 24],
        5: [b @ c ** 4 - 1 / 5, b @ (c * c * ac) - 1 / 10, b @ (c * acc) - 1 / 15, b @ (c * aac) - 1 / 30,
            b @ (ac * ac) - 1 / 20, b @ (a @ c ** 3) - 1 / 20, b @ (a @ (c * ac)) - 1 / 40,
            b @ (a @ acc) - 1 / 60, b @ (a @ aac) - 1 / 120],
    }
    return {p: max(abs(x) for x in v) for p, v in conds.items()}


@pytest.mark.parametrize("rk,order,embedded", [(4, 4, None), (5, 5, None), (45, 5, 4)])
def test_tableaux_satisfy_their_order_conditions(rk, order, embedded):
    """RK4 and the Fehlberg-5 weights of SBEs.h:395-416, and the Cash-Karp
    4(5) pair (J. R. Cash, A. H. Karp, ACM TOMS 16 (1990) 201, the method of
    the reference's RK-Methods/p201-cash.pdf): rows sum to c, the advancing
    weights reach the stated order and the embedded weights order 4 but not
    5, so their difference estimates the local error."""
    c, a, b, bs = pyoracle.tableau(rk)
    assert np.allclose(a.sum(1), c, atol=1e-15)
    assert np.all(np.triu(a) == 0)
    res = _order_conditions(c, a, b)
    assert all(res[p] < 1e-14 for p in range(1, order + 1)), res
    if order < 5:
        assert res[order + 1] > 1e-4, res
    if embedded:
        res = _order_conditions(c, a, bs)
        assert all(res[p] < 1e-14 for p in range(1, embedded + 1)), res
        assert res[embedded + 1] > 1e-5, res


def test_cashkarp_converges_to_the_reference_fine_solution():
    """The adaptive Cash-Karp extension has no counterpart in the reference;
    it is pinned by convergence: the reference's own fixed-step Fehlberg-5 at
    dt = 0.025 (harness build, N = 6 with dipoles, length gauge) is the fine
    solution, and Cash-Karp runs with an output interval of 0.5 (so the
    controller must cut the step) approach it as the tolerance tightens, below
    the error of the reference's own RK4 and Fehlberg-5 at that interval."""
    import copy

    fine = np.load(os.path.join(GOLDEN, "golden_synw6_w_rk5_fine.npz"))
    base = HARNESS_CASES["synw6_w_rk4"]
    errs, steps = {}, {}
    for rk, tol in (("rk4", None), ("rk5", None), ("cashkarp45", 1e-8), ("cashkarp45", 1e-10),
                    ("cashkarp45", 1e-12)):
        c = copy.deepcopy(base)
        c["calc"].update(rk=rk, dt=0.5)
        if tol:
            c["calc"]["tol"] = tol
        out = pyoracle.run(c)
        n = len(out["inter"])
        ref = fine["inter"][::20][:n]
        assert len(ref) == n
        errs[(rk, tol)] = _rel(out["inter"], ref)
        steps[(rk, tol)] = out["steps"]
    ck = [errs[("cashkarp45", t)] for t in (1e-8, 1e-10, 1e-12)]
    assert ck[0] > ck[1] > ck[2], errs
    assert ck[2] < 2e-10, errs
    assert ck[2] < errs[("rk5", None)] / 1000 and ck[2] < errs[("rk4", None)] / 1e5, errs
    assert steps[("cashkarp45", 1e-12)] > 2 * steps[("rk4", None)], steps
