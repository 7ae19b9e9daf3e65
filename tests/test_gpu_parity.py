"""GPU kernels against the CPU oracle (which is itself pinned to the
reference's outputs by test_oracle_golden.py).

Tolerances: the plain FP64 method must match to a relative 1e-10 of
max_t |J| on every current series (the stated parity bar), occupations to
1e-12 absolute.  Launch shape, steps per launch, CUDA graphs and batching
change nothing or only the summation order of the k-sum."""
import os

import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200.api import Solver
from cases import GOLDEN_CASES, variant
from oracle import pyoracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FP64_TOL = 1e-10


def rel(a, b):
    m = np.abs(b).max()
    return np.abs(a - b).max() / (m if m > 0 else 1.0)


def rel_series(a, b, scale):
    """max_t |a - b| / max_t |b| for one current series; a series that is
    zero up to rounding noise (e.g. the transverse intraband current of a
    linearly polarised pulse, ~1e-18) is measured against 1e-5 of the
    largest current of the run instead of against its own noise."""
    m = max(np.abs(b).max(), 1e-5 * scale)
    return np.abs(a - b).max() / m


_oracle_cache = {}


def oracle(name, case):
    if name not in _oracle_cache:
        _oracle_cache[name] = pyoracle.run(case)
    return _oracle_cache[name]


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_fp64_matches_oracle_and_reference(name):
    case = GOLDEN_CASES[name]
    out = ab.solve(case, precision="fp64")
    ref = oracle(name, case)
    gold = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    scale = max(np.abs(ref["inter"]).max(), np.abs(ref["intra"]).max())
    for key in ("inter", "intra"):
        for a in range(3):
            assert rel_series(getattr(out, key)[:, a], ref[key][:, a], scale) < FP64_TOL, (key, a)
            assert rel_series(getattr(out, key)[:, a], gold[key][:, a], scale) < FP64_TOL, (key, a)
    N = ref["dims"]["nband"]
    assert np.abs(out.occ[:, :N] - ref["occ"]).max() < 1e-12
    assert np.abs(out.occ - gold["occ_file"]).max() < 1e-12
    # coherence file: same flat-index element as the reference, last row 0
    assert np.abs(out.coh[:-1] - gold["coh_file"][:-1]).max() < 1e-12


def test_larger_grid_velocity_and_length_gauge():
    for gauge in ("Velocity", "Wannier"):
        case = variant(top__gauge=gauge, calc__Npoints=[37, 29], pulse__ellip=0.4, pulse__ncycles=3.0)
        out = ab.solve(case, precision="fp64")
        ref = pyoracle.run(case, nthreads=8)
        assert rel(out.inter, ref["inter"]) < FP64_TOL
        assert rel(out.intra, ref["intra"]) < FP64_TOL


@pytest.mark.parametrize("opts", [dict(tile_k=64), dict(tile_k=256), dict(tile_k=256, k_per_thread=2),
                                  dict(tile_k=96, k_per_thread=1)])
def test_launch_shape_only_reorders_the_k_sum(opts):
    case = variant(calc__Npoints=[23, 19])
    base = ab.solve(case, precision="fp64")
    out = ab.solve(case, precision="fp64", **opts)
    assert rel(out.inter, base.inter) < 1e-13
    assert rel(out.intra, base.intra) < 1e-13


@pytest.mark.parametrize("gauge,rk", [("Velocity", 5), ("Wannier", 4), ("Wannier", 5)])
def test_steps_per_launch_and_graph_are_bitwise_neutral(gauge, rk):
    """Both gauges carry the field at a step's end into the next step; a
    launch that starts at step s reads the same table entry."""
    case = variant(top__gauge=gauge, calc__Npoints=[16, 16], calc__RKorder=rk)
    a = ab.solve(case, precision="fp64", steps_per_launch=1024)
    b = ab.solve(case, precision="fp64", steps_per_launch=37)
    c = ab.solve(case, precision="fp64", steps_per_launch=100, use_graph=True)
    for x in (b, c):
        assert np.array_equal(x.inter, a.inter) and np.array_equal(x.intra, a.intra)
        assert np.array_equal(x.occ, a.occ)


def test_batch_equals_single_solves_bitwise():
    cases = [variant(calc__Npoints=[9 + i, 7 + 2 * i], pulse__cep=30.0 * i, Haldane__Mt2=1.0 + i,
                     pulse__ncycles=2.0 + i) for i in range(5)]
    cases.append(variant(top__gauge="Wannier", calc__Npoints=[11, 13]))
    probs = [ab.Problem.from_dict(c) for c in cases]
    singles = [ab.solve(p, precision="fp64") for p in probs]
    for graph in (False, True):
        b = ab.Batch(probs, precision="fp64", use_graph=graph, steps_per_launch=200)
        b.run()
        for i, s in enumerate(singles):
            o = b.get(i)
            assert np.array_equal(o.inter, s.inter) and np.array_equal(o.intra, s.intra), i
        b.close()


@pytest.mark.parametrize("gauge", ["Velocity", "Wannier"])
def test_packed_mixed_kernels_are_launch_split_neutral(gauge):
    """The packed mixed kernels carry FP32 increments between folds into the
    FP64 state (every 8 absolute steps) and keep an unfolded sum in the state
    at a launch's end, so where launches split the time loop changes no bit."""
    case = variant(top__gauge=gauge, calc__Npoints=[16, 16])
    shape = dict(precision="mixed", k_per_thread=2, tile_k=64)
    a = ab.solve(case, steps_per_launch=1024, **shape)
    for opts in (dict(steps_per_launch=37), dict(steps_per_launch=100, use_graph=True)):
        b = ab.solve(case, **shape, **opts)
        assert np.array_equal(b.inter, a.inter) and np.array_equal(b.intra, a.intra), opts
        assert np.array_equal(b.occ, a.occ), opts


@pytest.mark.parametrize("gauge", ["Velocity", "Wannier"])
def test_packed_and_scalar_mixed_kernels_agree(gauge):
    """Two k-points per thread (packed f32x2) and one (scalar FP32) do the same
    arithmetic up to FP32 operation order."""
    case = variant(top__gauge=gauge, calc__Npoints=[20, 18])
    a = ab.solve(case, precision="mixed", k_per_thread=1, tile_k=64)
    b = ab.solve(case, precision="mixed", k_per_thread=2, tile_k=128)
    scale = max(np.abs(a.inter).max(), np.abs(a.intra).max())
    for key in ("inter", "intra"):
        assert np.abs(getattr(a, key) - getattr(b, key)).max() < 1e-5 * scale, key


MIXED_TOL = 1e-3   # relative error per harmonic band, bands >= 1e-8 of the strongest


@pytest.mark.parametrize("gauge", ["Velocity", "Wannier"])
def test_mixed_precision_small_grid(gauge):
    """A small grid is the hard case: rounding noise averages over fewer k."""
    from antelope_b200.spectrum import per_harmonic_error

    case = variant(top__gauge=gauge, calc__Npoints=[31, 31], pulse__w0=0.0285, pulse__ncycles=4.0)
    a = ab.solve(case, precision="fp64")
    b = ab.solve(case, precision="mixed")
    orders, err, _ = per_harmonic_error({"inter": b.inter, "intra": b.intra},
                                        {"inter": a.inter, "intra": a.intra}, 0.1, 0.0285)
    assert len(orders) > 5
    assert err.max() < MIXED_TOL, (orders, err)


def test_mixed_precision_plain_method_config():
    """150x150 Haldane, 3.2 um 8-cycle sin^2 pulse, velocity gauge, RK4."""
    from antelope_b200 import workloads
    from antelope_b200.spectrum import per_harmonic_error

    a = ab.solve(workloads.haldane_case(150), precision="fp64")
    b = ab.solve(workloads.haldane_case(150), precision="mixed")
    orders, err, _ = per_harmonic_error({"inter": b.inter, "intra": b.intra},
                                        {"inter": a.inter, "intra": a.intra}, 0.1, 0.014238)
    assert len(orders) > 10
    assert err.max() < MIXED_TOL, (orders, err)


def test_server_alone_equals_in_mix():
    cases = [variant(calc__Npoints=[10 + i, 8 + i], pulse__ncycles=2.0 + 0.5 * i, pulse__cep=20.0 * i)
             for i in range(6)]
    probs = [ab.Problem.from_dict(c) for c in cases]
    alone = []
    srv = ab.Server(precision="fp64", steps_per_launch=128)
    for p in probs:
        rid = srv.submit(p)
        alone.append(srv.wait(rid, timeout=120)[0])
    ids = [srv.submit(p) for p in probs]
    for rid, a in zip(ids, alone):
        o, lat = srv.wait(rid, timeout=120)
        assert lat > 0
        assert np.array_equal(o.inter, a.inter) and np.array_equal(o.intra, a.intra)
    st = srv.stats()
    assert st["completed"] == 12 and st["failed"] == 0
    srv.close()


def test_server_cancel_and_single_delivery():
    """Requests cancelled in any state end CANCELLED and free their solve;
    the others complete with the same bits as alone; a request's final state
    is returned once, after which the server has forgotten it."""
    cases = [variant(calc__Npoints=[12 + i, 9], pulse__cep=15.0 * i) for i in range(20)]
    probs = [ab.Problem.from_dict(c) for c in cases]
    shape = dict(tile_k=64, k_per_thread=1)   # the server never tunes: fix the shape on both sides
    srv = ab.Server(precision="fp64", steps_per_launch=64, **shape)
    ids = [srv.submit(p) for p in probs]
    cancelled = set(ids[1::3])
    for rid in cancelled:
        srv.cancel(rid)
    for i, rid in enumerate(ids):
        if rid in cancelled:
            try:
                srv.wait(rid, timeout=120)   # may have finished before the cancel arrived
            except ab.SbeError as e:
                assert e.name == "SBE_CANCELLED"
        else:
            o, _ = srv.wait(rid, timeout=120)
            ref = ab.solve(probs[i], precision="fp64", steps_per_launch=64, **shape)
            assert np.array_equal(o.inter, ref.inter) and np.array_equal(o.occ, ref.occ)
    srv._problems[ids[0]] = probs[0]   # ask again for a delivered request
    with pytest.raises(ab.SbeError) as e:
        srv.wait(ids[0], timeout=1)
    assert "unknown request id" in str(e.value)
    st = srv.stats()
    assert st["failed"] == 0 and st["resident"] == 0
    srv.close()


def test_server_refuses_a_request_beyond_its_memory_budget():
    """Admission by device memory with a fixed budget (sbe_server_opts.
    mem_budget_bytes): a request that can never fit fails alone -- SBE_OOM with
    its own message -- while the requests around it, admitted as memory frees
    up, complete with the same bits as alone; failures do not leak into the
    rest of the stream."""
    shape = dict(tile_k=64, k_per_thread=1)
    small = [ab.Problem.from_dict(variant(calc__Npoints=[12 + i, 9], pulse__cep=15.0 * i)) for i in range(8)]
    big = ab.Problem.from_dict(variant(calc__Npoints=[400, 400]))
    srv = ab.Server(precision="fp64", steps_per_launch=64, mem_budget_bytes=2.0e6, **shape)
    ids = [srv.submit(p) for p in small[:4]]
    big_id = srv.submit(big)
    ids += [srv.submit(p) for p in small[4:]]
    with pytest.raises(ab.SbeError) as e:
        srv.wait(big_id, timeout=120)
    assert e.value.name == "SBE_OOM" and "admission refused" in str(e.value)
    for p, rid in zip(small, ids):
        o, _ = srv.wait(rid, timeout=120)
        ref = ab.solve(p, precision="fp64", steps_per_launch=64, **shape)
        assert np.array_equal(o.inter, ref.inter) and np.array_equal(o.occ, ref.occ)
    st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == len(small) and st["resident"] == 0
    srv.close()


def test_many_pulses_device_table_matches_host_table():
    """Ten pulses of every envelope kind: the field table the solver builds
    on the device agrees with the host-built one of sbe_solve_noalloc to the
    FP64 parity bar (the two evaluations of A(t) differ by about an ulp)."""
    from antelope_b200.api import solve_noalloc
    c = variant(calc__Npoints=[9, 8], calc__RKorder=5)
    envs = ["cos4", "gauss", "sin2", "cos4_clipped", "gauss_clipped"]
    c["laser"]["pulses"] = [{"E0": 0.001 + 0.0003 * i, "w0": 0.05 + 0.01 * i, "ncycles": 1.0 + 0.2 * i,
                             "ellip": 0.1 * (i % 3), "cep": 30.0 * i, "t0": 10.0 * i, "phix": 5.0 * i,
                             "env_name": envs[i % 5], "ncycles_clipped": 0.5} for i in range(10)]
    p = ab.Problem.from_dict(c)
    for prec, tol in (("fp64", FP64_TOL), ("mixed", 1e-6)):
        a = ab.solve(p, precision=prec, tile_k=64, k_per_thread=1)
        b = solve_noalloc(p, precision=prec, tile_k=64, k_per_thread=1)
        scale = max(np.abs(b.inter).max(), np.abs(b.intra).max())
        for key in ("inter", "intra"):
            for ax in range(2):
                assert rel_series(getattr(a, key)[:, ax], getattr(b, key)[:, ax], scale) < tol, (prec, key, ax)
        assert np.array_equal(a.laser, b.laser)


def test_cli_drop_in(tmp_path):
    """sbe_run in a directory holding inputParam.cfg writes the reference's
    six files with the reference's values."""
    import shutil
    import subprocess

    tdir = os.path.join(GOLDEN, "text_case")
    shutil.copy(os.path.join(tdir, "inputParam.cfg"), tmp_path / "inputParam.cfg")
    exe = os.path.join(os.path.dirname(ab.__file__), "bin", "sbe_run")
    subprocess.run([exe], cwd=tmp_path, check=True, capture_output=True)
    for f in ["interband_dipole_full_evol.dat", "intraband_current_full_evol.dat", "occupation__full__evol.dat"]:
        a = np.loadtxt(os.path.join(tdir, f))
        b = np.loadtxt(tmp_path / f)
        assert a.shape == b.shape
        assert rel(b, a) < FP64_TOL, f
    with open(os.path.join(tdir, "outlaserdata.dat"), "rb") as x, open(tmp_path / "outlaserdata.dat", "rb") as y:
        assert x.read() == y.read()
