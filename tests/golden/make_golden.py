"""Regenerate the golden fixtures of this folder from the reference itself.

Runs the unmodified reference (oracle/_ref/exec_hhg_ref, built by
``make -C oracle ref`` from the reference sources with the stand-in headers of
oracle/refshim) on every case of cases.GOLDEN_CASES, cases.MATERIAL_CASES,
cases.MULTIWSM_CASES and
cases.SNAPSHOT_CASES -- and the harness build (oracle/_ref/exec_hhg_harness, the
reference with the sin2 envelope and the SyntheticWannier material of
oracle/make_harness.py) on cases.HARNESS_CASES -- and stores its output files (snapshot files included) as
arrays in golden_<name>.npz; TEXT_CASE's files
are also kept verbatim in text_case/.
Usage:  python tests/golden/make_golden.py [case names]   (default: all)
"""
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import (GOLDEN_CASES, HARNESS_CASES, MATERIAL_CASES, MULTIWSM_CASES, SNAPSHOT_CASES,  # noqa: E402
                   TEXT_CASE)
from oracle import pyoracle  # noqa: E402
from antelope_b200 import cfgtext  # noqa: E402

FILES = ["interband_dipole_full_evol.dat", "intraband_current_full_evol.dat",
         "occupation__full__evol.dat", "coherence__full__evol.dat", "outlaserdata.dat"]


def main(names):
    cases = {**GOLDEN_CASES, **MATERIAL_CASES, **MULTIWSM_CASES, **SNAPSHOT_CASES, **HARNESS_CASES}
    for name in names or cases:
        with tempfile.TemporaryDirectory() as d:
            out = pyoracle.run_reference(cases[name], d, harness=name in HARNESS_CASES)
        np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)
        print(name, out["inter"].shape)
    if names:
        return
    tdir = os.path.join(HERE, "text_case")
    os.makedirs(tdir, exist_ok=True)
    with tempfile.TemporaryDirectory() as d:
        pyoracle.run_reference(TEXT_CASE, d)
        for f in FILES + ["inputParam.cfg"]:
            shutil.copy(os.path.join(d, f), os.path.join(tdir, f))
    with open(os.path.join(tdir, "inputParam.cfg")) as f:
        assert f.read() == cfgtext.dumps(TEXT_CASE)


if __name__ == "__main__":
    main(sys.argv[1:])
