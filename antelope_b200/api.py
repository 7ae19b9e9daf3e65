"""Python front end of the native library (include/sbe.h).

``Problem`` wraps an inputParam.cfg; ``solve`` runs one problem through the
GPU solver; ``Batch`` runs many at once; ``Server`` is the continuous-
batching request loop.  Output arrays have the reference's file layout.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import cfgtext
from .capi import COutputs, Dims, Opts, P, ServerOpts, STATUS, lib


class SbeError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status
        self.name = STATUS.get(status, str(status))


def _check(st: int):
    if st != 0:
        raise SbeError(st, lib.sbe_last_error_message().decode(errors="replace"))


def _opts(precision=None, tile_k=0, k_per_thread=0, steps_per_launch=0, use_graph=False, device=0,
          profile=False):
    o = Opts()
    lib.sbe_opts_default(C.byref(o))
    o.device = device
    o.precision = -1 if precision is None else {"fp64": 0, "mixed": 1, 0: 0, 1: 1}[precision]
    o.tile_k, o.k_per_thread, o.steps_per_launch = tile_k, k_per_thread, steps_per_launch
    o.use_graph = 1 if use_graph else 0
    o.profile = 1 if profile else 0
    return o


def _kernel_times(fn, h):
    pm, rm = C.c_double(0), C.c_double(0)
    pn, rn = C.c_int(0), C.c_int(0)
    _check(fn(h, C.byref(pm), C.byref(pn), C.byref(rm), C.byref(rn)))
    return {"propagate_ms": pm.value, "propagate_launches": pn.value, "reduce_ms": rm.value,
            "reduce_launches": rn.value}


@dataclass
class Outputs:
    inter: np.ndarray   # [Nt, 3]
    intra: np.ndarray   # [Nt, 3]
    occ: np.ndarray     # [Nt, N+1]
    coh: np.ndarray     # [Nt, 2]
    laser: np.ndarray   # [Nt, 7]

    @classmethod
    def empty(cls, dims: Dims):
        Nt, N = dims.Nt, dims.nband
        return cls(np.zeros((Nt, 3)), np.zeros((Nt, 3)), np.zeros((Nt, N + 1)), np.zeros((Nt, 2)),
                   np.zeros((Nt, 7)))

    def c(self) -> COutputs:
        return COutputs(*(a.ctypes.data for a in (self.inter, self.intra, self.occ, self.coh, self.laser)))


class Problem:
    """An inputParam.cfg, parsed by the native library."""

    def __init__(self, handle):
        self._h = handle
        d = Dims()
        _check(lib.sbe_problem_dims(self._h, C.byref(d)))
        self.dims = d

    @classmethod
    def from_cfg(cls, path: str) -> "Problem":
        h = P()
        _check(lib.sbe_problem_from_cfg(os.fsencode(path), C.byref(h)))
        return cls(h)

    @classmethod
    def from_text(cls, text: str) -> "Problem":
        h = P()
        _check(lib.sbe_problem_from_string(text.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_dict(cls, case: dict) -> "Problem":
        return cls.from_text(cfgtext.dumps(case))

    @property
    def Nt(self):
        return self.dims.Nt

    @property
    def ntotal(self):
        return self.dims.ntotal

    def laser(self) -> np.ndarray:
        out = np.zeros((self.dims.Nt, 7))
        _check(lib.sbe_problem_laser(self._h, out.ctypes.data))
        return out

    def model_tables(self) -> dict:
        """The tight-binding tables of a table model (``sbe_problem_model``):
        vectors [nvec, 2], h [nvec, N, N], optional d / j [nvec, 2, N, N]
        (complex), the material's Brillouin-zone axes bz [9], nband, nval."""
        from .capi import Model
        m = Model()
        _check(lib.sbe_problem_model(self._h, C.byref(m)))
        N, nv = m.nband, m.nvec
        out = {"nband": N, "nval": m.nval, "vec": np.zeros((nv, 2)), "h": np.zeros((nv, N, N), complex),
               "d": np.zeros((nv, 2, N, N), complex) if m.has_dipoles else None,
               "j": np.zeros((nv, 2, N, N), complex) if m.has_current_tables else None, "bz": np.zeros(9)}
        m.vec, m.h, m.bz = out["vec"].ctypes.data, out["h"].ctypes.data, out["bz"].ctypes.data
        if out["d"] is not None:
            m.d = out["d"].ctypes.data
        if out["j"] is not None:
            m.j = out["j"].ctypes.data
        _check(lib.sbe_problem_model(self._h, C.byref(m)))
        return out

    def snapshot_dims(self) -> dict:
        """Snapshot interval (steps), number of snapshots and Npoints[0]
        (``sbe_problem_snapshots``; zeros when calc.shotNumber <= 0)."""
        v = [C.c_int() for _ in range(3)]
        _check(lib.sbe_problem_snapshots(self._h, *[C.byref(x) for x in v]))
        return {"interval": v[0].value, "nshots": v[1].value, "n0": v[2].value}

    def __del__(self):
        if getattr(self, "_h", None):
            lib.sbe_problem_destroy(self._h)
            self._h = None


def _snapshot_arrays(problem: "Problem", nk: int):
    sd = problem.snapshot_dims()
    ns = sd["nshots"]
    return (np.zeros((ns, sd["n0"])), np.zeros((ns, nk)), np.zeros((ns, nk), dtype=np.complex128))


def write_snapshots(problem: "Problem", snaps: dict, out_dir: str):
    """The reference's snapshot files from ``snapshots()`` arrays
    (``sbe_write_snapshots``)."""
    occ1d = np.ascontiguousarray(snaps["occ1d"], dtype=np.float64)
    nc = np.ascontiguousarray(snaps["nc"], dtype=np.float64)
    pi = np.ascontiguousarray(snaps["pi"], dtype=np.complex128)
    _check(lib.sbe_write_snapshots(problem._h, occ1d.ctypes.data, nc.ctypes.data, pi.ctypes.data,
                                   os.fsencode(out_dir)))


class Solver:
    """One solve on the GPU (``sbe_solver_*``); ``k_slice=(k_begin, k_end)``
    restricts it to a block of the k-grid (``sbe_solver_create_slice``)."""

    def __init__(self, problem: Problem, k_slice: tuple[int, int] | None = None, **opts):
        self.problem = problem
        self._k_slice = k_slice
        self._h = P()
        if k_slice is None:
            _check(lib.sbe_solver_create(problem._h, C.byref(_opts(**opts)), C.byref(self._h)))
        else:
            _check(lib.sbe_solver_create_slice(problem._h, C.byref(_opts(**opts)), int(k_slice[0]),
                                               int(k_slice[1]), C.byref(self._h)))

    def run(self, stream: int = 0):
        _check(lib.sbe_solver_run(self._h, C.c_void_p(stream)))

    def get(self, out: Outputs | None = None) -> Outputs:
        out = out or Outputs.empty(self.problem.dims)
        _check(lib.sbe_solver_get(self._h, C.byref(out.c())))
        return out

    @property
    def launches(self) -> int:
        return lib.sbe_solver_launches(self._h)

    def kernel_times(self) -> dict:
        return _kernel_times(lib.sbe_solver_kernel_times, self._h)

    def sums(self) -> np.ndarray:
        """Per-step k-sums of this solver's k-points, (Nt + 1) x width,
        additive over k-slices (``sbe_solver_sums``)."""
        out = np.zeros((self.problem.dims.Nt + 1, lib.sbe_sums_width(self.problem._h)))
        _check(lib.sbe_solver_sums(self._h, out.ctypes.data))
        return out

    def snapshots(self) -> dict:
        """Density snapshots of the finished run (``sbe_solver_snapshots``):
        occ1d [nshots, Npoints[0]], per-k nc [nshots, nk] and pi [nshots, nk]
        (complex)."""
        nk = self._k_slice[1] - self._k_slice[0] if self._k_slice else self.problem.ntotal
        occ1d, nc, pi = _snapshot_arrays(self.problem, nk)
        _check(lib.sbe_solver_snapshots(self._h, occ1d.ctypes.data, nc.ctypes.data, pi.ctypes.data))
        return {"occ1d": occ1d, "nc": nc, "pi": pi}

    def harmonics(self, w0: float, hmax: int) -> np.ndarray:
        """Band powers of harmonic orders 1..hmax, computed on the GPU
        (``sbe_solver_harmonics``; the analysis-script convention)."""
        out = np.zeros(hmax)
        _check(lib.sbe_solver_harmonics(self._h, C.c_double(w0), hmax, out.ctypes.data))
        return out

    def steps(self) -> dict:
        """Accepted steps, attempts and rejected attempts of the finished run."""
        v = [C.c_longlong() for _ in range(3)]
        _check(lib.sbe_solver_steps(self._h, *[C.byref(x) for x in v]))
        return {"steps": v[0].value, "attempts": v[1].value, "rejects": v[2].value}

    def close(self):
        if getattr(self, "_h", None):
            lib.sbe_solver_destroy(self._h)
            self._h = None

    __del__ = close


def assemble(problem: Problem, sums: np.ndarray) -> "Outputs":
    """Output arrays from k-sums added over all slices (``sbe_assemble``,
    host only)."""
    sums = np.ascontiguousarray(sums, dtype=np.float64)
    if sums.shape != (problem.dims.Nt + 1, lib.sbe_sums_width(problem._h)):
        raise ValueError("sums has the wrong shape")
    out = Outputs.empty(problem.dims)
    _check(lib.sbe_assemble(problem._h, sums.ctypes.data, C.byref(out.c())))
    return out


def solve(problem, **opts) -> Outputs:
    """Run one problem (a Problem, a cfg path or a case dict) to completion."""
    if isinstance(problem, dict):
        problem = Problem.from_dict(problem)
    elif isinstance(problem, (str, os.PathLike)):
        problem = Problem.from_cfg(problem)
    s = Solver(problem, **opts)
    try:
        s.run()
        return s.get()
    finally:
        s.close()


def solve_noalloc(problem: Problem, stream: int = 0, **opts) -> Outputs:
    """Allocation-free solve (``sbe_solve_noalloc``): the library allocates no
    device memory for it; working memory is a fixed array inside the library."""
    out = Outputs.empty(problem.dims)
    _check(lib.sbe_solve_noalloc(problem._h, C.byref(_opts(**opts)), C.c_void_p(stream), C.byref(out.c())))
    return out


def run_cfg(cfg_path: str, out_dir: str = ".", **opts):
    """The drop-in: read an inputParam.cfg, solve, write the reference's files."""
    _check(lib.sbe_run_cfg(os.fsencode(cfg_path), os.fsencode(out_dir), C.byref(_opts(**opts))))


def write_outputs(problem: Problem, out: Outputs, out_dir: str):
    _check(lib.sbe_write_outputs(problem._h, C.byref(out.c()), os.fsencode(out_dir)))


class Batch:
    """Many solves advanced together (``sbe_batch_*``)."""

    def __init__(self, problems: list[Problem], **opts):
        self.problems = list(problems)
        arr = (P * len(self.problems))(*[p._h for p in self.problems])
        self._h = P()
        _check(lib.sbe_batch_create(arr, len(self.problems), C.byref(_opts(**opts)), C.byref(self._h)))

    def run(self, stream: int = 0):
        _check(lib.sbe_batch_run(self._h, C.c_void_p(stream)))

    def get(self, i: int) -> Outputs:
        out = Outputs.empty(self.problems[i].dims)
        _check(lib.sbe_batch_get(self._h, i, C.byref(out.c())))
        return out

    def snapshots(self, i: int) -> dict:
        """Density snapshots of solve i (``sbe_batch_snapshots``)."""
        occ1d, nc, pi = _snapshot_arrays(self.problems[i], self.problems[i].ntotal)
        _check(lib.sbe_batch_snapshots(self._h, i, occ1d.ctypes.data, nc.ctypes.data, pi.ctypes.data))
        return {"occ1d": occ1d, "nc": nc, "pi": pi}

    def harmonics(self, i: int, w0: float, hmax: int) -> np.ndarray:
        """Band powers of harmonic orders 1..hmax of solve i, on the GPU."""
        out = np.zeros(hmax)
        _check(lib.sbe_batch_harmonics(self._h, i, C.c_double(w0), hmax, out.ctypes.data))
        return out

    def steps(self, i: int) -> dict:
        """Accepted steps, attempts and rejected attempts of solve i."""
        v = [C.c_longlong() for _ in range(3)]
        _check(lib.sbe_batch_steps(self._h, i, *[C.byref(x) for x in v]))
        return {"steps": v[0].value, "attempts": v[1].value, "rejects": v[2].value}

    @property
    def launches(self) -> int:
        return lib.sbe_batch_launches(self._h)

    def kernel_times(self) -> dict:
        return _kernel_times(lib.sbe_batch_kernel_times, self._h)

    def close(self):
        if getattr(self, "_h", None):
            lib.sbe_batch_destroy(self._h)
            self._h = None

    __del__ = close


class Server:
    """Continuous-batching request loop (``sbe_server_*``)."""

    def __init__(self, precision=None, steps_per_launch=0, max_resident=0, mem_budget_bytes=0.0,
                 tile_k=0, k_per_thread=0, device=0):
        o = ServerOpts()
        o.device = device
        o.precision = -1 if precision is None else {"fp64": 0, "mixed": 1}[precision]
        o.steps_per_launch, o.max_resident, o.mem_budget_bytes = steps_per_launch, max_resident, mem_budget_bytes
        o.tile_k, o.k_per_thread = tile_k, k_per_thread
        self._h = P()
        self._problems = {}
        _check(lib.sbe_server_create(C.byref(o), C.byref(self._h)))

    def submit(self, problem: Problem) -> int:
        rid = C.c_longlong(0)
        _check(lib.sbe_server_submit(self._h, problem._h, C.byref(rid)))
        self._problems[rid.value] = problem
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0):
        """Outputs and latency of a request.  Its final state is returned once
        (the server then forgets the request); a timeout leaves it waitable."""
        prob = self._problems[rid]
        out = Outputs.empty(prob.dims)
        lat = C.c_double(0.0)
        st = lib.sbe_server_wait(self._h, rid, float(timeout), C.byref(out.c()), C.byref(lat))
        if STATUS.get(st) != "SBE_TIMEOUT":
            self._problems.pop(rid, None)
        _check(st)
        return out, lat.value

    def cancel(self, rid: int):
        _check(lib.sbe_server_cancel(self._h, rid))

    def stats(self) -> dict:
        c = (C.c_longlong * 5)()
        _check(lib.sbe_server_stats(self._h, c))
        return dict(zip(("submitted", "completed", "failed", "resident", "launches"), list(c)))

    def close(self):
        if getattr(self, "_h", None):
            lib.sbe_server_destroy(self._h)
            self._h = None

    __del__ = close


def measure_fma_peaks(device: int = 0):
    """(fp64, fp32, packed f32x2) FMA-chain peaks in TFLOP/s."""
    a, b, c = C.c_double(0), C.c_double(0), C.c_double(0)
    _check(lib.sbe_measure_fma_peaks(device, C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value
