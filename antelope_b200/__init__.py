"""B200-native propagator of the Semiconductor Bloch Equations.

Drop-in for the time propagation of ftachacon/antelope (src/GeneralModel):
same inputParam.cfg, same output arrays/files.  The computation lives in the
native library ``libsbe_b200.so`` (C ABI: include/sbe.h), built from
antelope_b200/csrc by ``antelope_b200.build``; this package is a thin ctypes
front end.  There is no Python or CPU fallback: if the library is missing the
import of ``antelope_b200.capi`` raises.
"""
from .api import (Batch, Outputs, Problem, SbeError, Server, measure_fma_peaks,  # noqa: F401
                  run_cfg, solve)
