"""Density snapshots (calc.shotNumber, antelope.cpp:267-422) on the GPU.

Every int(period0 / shotNumber / dt) steps the kernels store each k-point's
conduction occupation and coherence after the step (band basis in the
velocity gauge, eigenbasis of H0(k + A(t_n)) in the length gauge), and a
second kernel forms the 1-D integrated occupation.  Checked against the CPU
oracle (pinned to the reference's snapshot files by test_oracle_golden.py)
and against the reference's files themselves where they are defined (the
last k-point: its loop reads every other entry through a stale index).
The coherence carries the eigenvector phases (zheevr's in the reference,
closed-form spinors here), so its modulus is compared.

Tolerances: plain FP64 to 1e-10 of the largest value; the mixed method to
1e-5 of it (FP32 stages, FP64 state)."""
import os

import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200.api import Batch, Solver
from cases import SNAPSHOT_CASES, variant
from oracle import pyoracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
HALDANE_SHOTS = ["vg_shots", "lw_shots", "vg_shots_fermi_t1"]
TABLE_SHOTS = ["kanemele_w_shots", "tmdcs_v_shots"]   # N-band kernels, both gauges


def _run(case, **opts):
    s = Solver(ab.Problem.from_dict(case), **opts)
    s.run()
    out, snaps = s.get(), s.snapshots()
    s.close()
    return out, snaps


def _close(a, b, tol):
    return np.abs(a - b).max() <= tol * np.abs(b).max()


@pytest.mark.parametrize("name", HALDANE_SHOTS + TABLE_SHOTS)
def test_fp64_snapshots_match_oracle_and_reference(name):
    case = SNAPSHOT_CASES[name]
    _, snaps = _run(case, precision="fp64")
    ref = pyoracle.run(case)
    gold = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    ns, nt = ref["nc"].shape
    assert snaps["nc"].shape == (ns, nt) and snaps["occ1d"].shape == ref["occ1d"].shape
    assert _close(snaps["occ1d"], ref["occ1d"], 1e-10)
    assert _close(snaps["nc"], ref["nc"], 1e-10)
    assert _close(np.abs(snaps["pi"]), np.abs(ref["pi"]), 1e-10)
    # the reference's own files: the 1-D integration (printed to 7 digits)
    # and the entry of the last k-point
    floor = 1e-13 * np.abs(gold["occ1d"]).max()
    assert np.all(np.abs(snaps["occ1d"] - gold["occ1d"]) <= 6e-7 * np.abs(gold["occ1d"]) + floor)
    rn, rp = gold["nc"].reshape(ns, nt), gold["pi"].reshape(ns, nt)
    assert np.abs(snaps["nc"][:, -1] - rn[:, -1]).max() <= 1e-10 * np.abs(rn).max()
    assert np.abs(np.abs(snaps["pi"][:, -1]) - np.abs(rp[:, -1])).max() <= 1e-10 * np.abs(rp[:, -1]).max()


@pytest.mark.parametrize("name", HALDANE_SHOTS + TABLE_SHOTS)
def test_mixed_snapshots_near_fp64(name):
    case = SNAPSHOT_CASES[name]
    _, a = _run(case, precision="fp64")
    _, b = _run(case, precision="mixed")
    assert _close(b["occ1d"], a["occ1d"], 1e-5)
    assert _close(b["nc"], a["nc"], 1e-5)
    assert _close(np.abs(b["pi"]), np.abs(a["pi"]), 1e-5)


@pytest.mark.parametrize("name,prec,kpt", [("vg_shots", "fp64", 1), ("vg_shots", "fp64", 2),
                                           ("vg_shots", "mixed", 2), ("lw_shots", "fp64", 1),
                                           ("lw_shots", "mixed", 1)])
def test_snapshots_independent_of_launch_split_graphs_and_batching(name, prec, kpt):
    """Steps per launch, CUDA graphs and batching leave the snapshots bitwise
    unchanged (same tiling); the snapshot steps need not align with launches."""
    case = SNAPSHOT_CASES[name]
    shape = dict(precision=prec, tile_k=64 * kpt, k_per_thread=kpt)
    _, a = _run(case, steps_per_launch=1024, **shape)
    _, b = _run(case, steps_per_launch=37, use_graph=True, **shape)
    for key in ("occ1d", "nc", "pi"):
        assert np.array_equal(a[key], b[key]), key
    other = ab.Problem.from_dict(variant(calc__Npoints=[9, 5]))
    bt = Batch([other, ab.Problem.from_dict(case)], steps_per_launch=100, **shape)
    bt.run()
    c = bt.snapshots(1)
    with pytest.raises(ab.SbeError):
        bt.snapshots(0)   # no snapshots asked for
    bt.close()
    for key in ("occ1d", "nc", "pi"):
        assert np.array_equal(a[key], c[key]), key


def test_snapshots_of_k_slices_add_up():
    """A k-slice holds its k-points' values and its part of the 1-D sums."""
    case = SNAPSHOT_CASES["lw_shots"]
    p = ab.Problem.from_dict(case)
    _, whole = _run(case, precision="fp64")
    cut = 17
    parts = []
    for sl in ((0, cut), (cut, p.ntotal)):
        s = Solver(p, k_slice=sl, precision="fp64")
        s.run()
        parts.append(s.snapshots())
        s.close()
    assert np.abs(np.concatenate([parts[0]["nc"], parts[1]["nc"]], axis=1) - whole["nc"]).max() < 1e-12
    assert _close(parts[0]["occ1d"] + parts[1]["occ1d"], whole["occ1d"], 1e-12)


def test_run_cfg_writes_snapshot_files(tmp_path):
    case = SNAPSHOT_CASES["vg_shots"]
    cfg = tmp_path / "inputParam.cfg"
    from antelope_b200 import cfgtext
    cfg.write_text(cfgtext.dumps(case))
    ab.run_cfg(str(cfg), str(tmp_path))
    got = pyoracle.read_outputs(str(tmp_path))
    ref = pyoracle.run(case)
    floor = 1e-13 * np.abs(ref["occ1d"]).max()
    assert np.all(np.abs(got["occ1d"] - ref["occ1d"]) <= 6e-7 * np.abs(ref["occ1d"]) + floor)
    assert _close(got["nc"], ref["nc"].ravel(), 1e-10)
    assert (tmp_path / "snapshot_log.dat").exists()


def test_solver_without_snapshots_refuses_to_return_them():
    s = Solver(ab.Problem.from_dict(variant()), precision="fp64")
    s.run()
    with pytest.raises(ab.SbeError) as e:
        s.snapshots()
    s.close()
    assert "no snapshots" in str(e.value)


def test_adaptive_table_model_snapshots_match_oracle():
    """Cash-Karp 4(5) steps (one step size per solve, steps landing on the
    output times): the snapshot of output step n is taken once the accepted
    steps reach t_{n+1}."""
    from antelope_b200 import wannier
    case = wannier.wannier_case(seed=3, n=9, ncycles=0.05, rk="cashkarp45", tol=1e-9)
    case["calc"]["shotNumber"] = 100
    _, snaps = _run(case, precision="fp64")
    ref = pyoracle.run(case)
    assert snaps["nc"].shape == ref["nc"].shape and snaps["nc"].shape[0] > 2
    # adaptive steps: the step sequence is the oracle's to rounding, the
    # values to the controller's tolerance
    assert _close(snaps["occ1d"], ref["occ1d"], 1e-7)
    assert _close(snaps["nc"], ref["nc"], 1e-7)
    assert _close(np.abs(snaps["pi"]), np.abs(ref["pi"]), 1e-7)
