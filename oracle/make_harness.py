"""Generate the harness variant of the reference build (test infrastructure).

The reference has no ``sin2`` envelope and no material with dipole matrices
that it can compile (Materials/Wannier90.h includes a header missing from the
reference tree, and SBEs.h:211-214 keeps its construction commented out).  To
run the reference's own propagation code on those inputs, this script writes
build-time copies of three reference files into an output folder (never into
the reference tree, never into the repository's history) with small anchored
insertions:

  SBEs.h       + ``#include "SyntheticWannier.h"`` after the material list
                 (SBEs.h:30) and one more branch of the material dispatch
                 (SBEs.h:167-215): target "SyntheticWannier" constructs the
                 harness material of oracle/refharness/SyntheticWannier.h;
  laser.h      + the envelope "sin2", f(t) = cos^2(w0 t / (2 N)) on
                 |t| <= N T / 2 with its analytic derivative (the same support
                 and argument scale as "cos4", laser.h:77-105, 150-158);
  antelope.cpp   copied unchanged, so that its quoted includes resolve to the
                 two files above first.

Every insertion is anchored on text that must occur exactly once; if the
reference changes and an anchor is missing the script fails.  Usage:

  python3 oracle/make_harness.py <reference src/GeneralModel> <output dir>
"""
import os
import sys


def insert(text: str, anchor: str, new: str, where: str = "after") -> str:
    n = text.count(anchor)
    if n != 1:
        raise SystemExit(f"make_harness: anchor found {n} times, expected once: {anchor!r}")
    i = text.index(anchor)
    j = i + len(anchor) if where == "after" else i
    return text[:j] + new + text[j:]


SBES_INCLUDE = '\n#include "SyntheticWannier.h"   // harness material (oracle/refharness)\n'

SBES_BRANCH = '''    else if (targetMaterial == "SyntheticWannier")   // harness-only branch
    {
        material = new SyntheticWannier( &cfg[targetMaterial.c_str()] );
    }
'''

LASER_ENUM = ",\n    ENVELOPE_SIN2   // harness-only: cos^2 envelope"

LASER_NAME = '\n        else if (envname == "sin2") {envtype = ENVELOPE_SIN2;}   // harness-only'

LASER_WIDTH = '''        case ENVELOPE_SIN2:   // harness-only: support N T / 2 each side, as cos4
            twidth = ncycles*period0/2;
            envfactor = w0/(2*ncycles);
            break;
'''

LASER_VALUE = '''        case ENVELOPE_SIN2:   // harness-only: f = cos^2(t w0 / (2N)), f' = -2 w0/(2N) sin cos
            if (std::fabs(_t) > twidth) return 0;
            if (_isDt) return -2.* envfactor *sin(_t* envfactor) * cos(_t* envfactor);
            else return cos(_t* envfactor) * cos(_t* envfactor);

'''


def main(src: str, out: str) -> None:
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(src, "SBEs.h")) as f:
        sbes = f.read()
    sbes = insert(sbes, '#include "system_list.h"', SBES_INCLUDE)
    # the dispatch's final branch is the `else` that reports an unknown material
    tail = '    else\n    {\n        std::cerr << "Undefined Material\\n";'
    sbes = insert(sbes, tail, SBES_BRANCH, where="before")

    with open(os.path.join(src, "laser.h")) as f:
        laser = f.read()
    laser = insert(laser, "    ENVELOPE_COS4_CLIPPED", LASER_ENUM)
    laser = insert(laser, 'else if (envname == "cos4_clipped") {envtype = ENVELOPE_COS4_CLIPPED;}', LASER_NAME)
    laser = insert(laser, "        // clipped part give additional length\n", LASER_WIDTH, where="before")
    laser = insert(laser, "        case ENVELOPE_COS4_CLIPPED:\n            if (abs(_t) > twidth) return 0;",
                   LASER_VALUE, where="before")

    with open(os.path.join(src, "antelope.cpp")) as f:
        driver = f.read()
    for name, text in (("SBEs.h", sbes), ("laser.h", laser), ("antelope.cpp", driver)):
        with open(os.path.join(out, name), "w") as f:
            f.write(text)


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2])
