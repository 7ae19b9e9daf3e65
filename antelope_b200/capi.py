"""ctypes binding of include/sbe.h (libsbe_b200.so).

Loading fails loudly when the native library has not been built: the
product has no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbe_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "sbe.h")

STATUS = {0: "SBE_OK", 1: "SBE_BAD_CONFIG", 2: "SBE_UNSUPPORTED", 3: "SBE_OOM", 4: "SBE_CUDA_ERROR",
          5: "SBE_TIMEOUT", 6: "SBE_CANCELLED", 7: "SBE_INVALID_ARGUMENT", 8: "SBE_NOT_READY"}


class Dims(C.Structure):
    _fields_ = [("Nt", C.c_int), ("nband", C.c_int), ("nval", C.c_int), ("ntotal", C.c_int),
                ("Nk", C.c_int * 3), ("gauge", C.c_int), ("rk", C.c_int), ("precision", C.c_int),
                ("model", C.c_int), ("inter_intra", C.c_int), ("atmin", C.c_double), ("dt", C.c_double),
                ("dV", C.c_double), ("total_weight", C.c_double)]


class Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("tile_k", C.c_int),
                ("k_per_thread", C.c_int), ("steps_per_launch", C.c_int), ("use_graph", C.c_int),
                ("profile", C.c_int)]


class Model(C.Structure):
    _fields_ = [("nband", C.c_int), ("nval", C.c_int), ("nvec", C.c_int), ("has_dipoles", C.c_int),
                ("has_current_tables", C.c_int)] + [(n, C.c_void_p) for n in ("vec", "h", "d", "j", "bz")]


class COutputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("inter", "intra", "occ", "coh", "laser")]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("steps_per_launch", C.c_int),
                ("max_resident", C.c_int), ("mem_budget_bytes", C.c_double), ("tile_k", C.c_int),
                ("k_per_thread", C.c_int)]


P = C.c_void_p


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m antelope_b200.build` "
                          "(or __graft_entry__.build()) first")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "sbe_abi_version": (C.c_int, []),
        "sbe_last_error_message": (C.c_char_p, []),
        "sbe_opts_default": (None, [C.POINTER(Opts)]),
        "sbe_problem_from_cfg": (C.c_int, [C.c_char_p, C.POINTER(P)]),
        "sbe_problem_from_string": (C.c_int, [C.c_char_p, C.POINTER(P)]),
        "sbe_problem_dims": (C.c_int, [P, C.POINTER(Dims)]),
        "sbe_problem_laser": (C.c_int, [P, C.c_void_p]),
        "sbe_problem_model": (C.c_int, [P, C.POINTER(Model)]),
        "sbe_problem_snapshots": (C.c_int, [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "sbe_problem_destroy": (None, [P]),
        "sbe_solver_snapshots": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_void_p]),
        "sbe_batch_snapshots": (C.c_int, [P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
        "sbe_write_snapshots": (C.c_int, [P, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p]),
        "sbe_solver_create": (C.c_int, [P, C.POINTER(Opts), C.POINTER(P)]),
        "sbe_solver_run": (C.c_int, [P, C.c_void_p]),
        "sbe_solver_get": (C.c_int, [P, C.POINTER(COutputs)]),
        "sbe_solver_launches": (C.c_int, [P]),
        "sbe_solver_harmonics": (C.c_int, [P, C.c_double, C.c_int, C.c_void_p]),
        "sbe_solver_create_slice": (C.c_int, [P, C.POINTER(Opts), C.c_int, C.c_int, C.POINTER(P)]),
        "sbe_sums_width": (C.c_int, [P]),
        "sbe_solver_sums": (C.c_int, [P, C.c_void_p]),
        "sbe_assemble": (C.c_int, [P, C.c_void_p, C.POINTER(COutputs)]),
        "sbe_batch_harmonics": (C.c_int, [P, C.c_int, C.c_double, C.c_int, C.c_void_p]),
        "sbe_solver_steps": (C.c_int, [P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                       C.POINTER(C.c_longlong)]),
        "sbe_solver_destroy": (None, [P]),
        "sbe_solver_kernel_times": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                              C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "sbe_batch_kernel_times": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                             C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "sbe_write_outputs": (C.c_int, [P, C.POINTER(COutputs), C.c_char_p]),
        "sbe_run_cfg": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Opts)]),
        "sbe_batch_create": (C.c_int, [C.POINTER(P), C.c_int, C.POINTER(Opts), C.POINTER(P)]),
        "sbe_batch_run": (C.c_int, [P, C.c_void_p]),
        "sbe_batch_get": (C.c_int, [P, C.c_int, C.POINTER(COutputs)]),
        "sbe_batch_launches": (C.c_int, [P]),
        "sbe_batch_steps": (C.c_int, [P, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_longlong)]),
        "sbe_batch_destroy": (None, [P]),
        "sbe_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(P)]),
        "sbe_server_submit": (C.c_int, [P, P, C.POINTER(C.c_longlong)]),
        "sbe_server_wait": (C.c_int, [P, C.c_longlong, C.c_double, C.POINTER(COutputs),
                                      C.POINTER(C.c_double)]),
        "sbe_server_cancel": (C.c_int, [P, C.c_longlong]),
        "sbe_server_stats": (C.c_int, [P, C.POINTER(C.c_longlong)]),
        "sbe_server_destroy": (None, [P]),
        "sbe_solve_noalloc": (C.c_int, [P, C.POINTER(Opts), C.c_void_p, C.POINTER(COutputs)]),
        "sbe_measure_fma_peaks": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                             C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def declared_functions() -> list[str]:
    """Function names declared in include/sbe.h (for the export check)."""
    import re

    with open(HEADER) as f:
        text = f.read()
    return sorted(set(re.findall(r"\b(sbe_[a-z0-9_]+)\s*\(", text)))
