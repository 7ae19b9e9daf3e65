"""B200-native propagator of the Semiconductor Bloch Equations.

Drop-in for the time propagation of ftachacon/antelope (src/GeneralModel):
same inputParam.cfg, same output arrays/files.  The computation lives in the
native library ``libsbe_b200.so`` (C ABI: include/sbe.h), built from
antelope_b200/csrc by ``antelope_b200.build``; this package is a thin ctypes
front end.  There is no Python or CPU fallback: the first use of the solver
API (``antelope_b200.Problem``, ``solve``, ...) loads the library and raises
if it is missing.  The helper modules that need no GPU -- ``cfgtext`` (the
inputParam.cfg text format), ``workloads`` (the synthetic benchmark inputs),
``wannier`` (synthetic tight-binding tables), ``spectrum`` and ``dist`` -- can
be imported without loading it.
"""
_API = ("Batch", "Outputs", "Problem", "SbeError", "Server", "measure_fma_peaks", "run_cfg", "solve")


def __getattr__(name):
    if name in _API:
        from . import api
        return getattr(api, name)
    raise AttributeError(f"module 'antelope_b200' has no attribute {name!r}")


def __dir__():
    return sorted(list(globals()) + list(_API))
