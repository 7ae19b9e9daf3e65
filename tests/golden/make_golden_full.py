"""Regenerate the full-size golden fixtures (full_*.npz) from the reference.

The small cases of make_golden.py run in about a second; these run the
reference on the Haldane configuration at its own size -- 150 x 150 k-points,
the 3.2 um 8-cycle pulse, dt = 0.1 (35 303 steps), RK4, T2 = 220 -- so that
parity is also shown over the full number of time steps:

  full_c1_vg_cos4     velocity gauge, cos4 envelope (the unmodified reference)
  full_c1_lw_cos4     length gauge, cos4 envelope (the unmodified reference)
  full_c1_vg_sin2     velocity gauge, sin2 envelope (the harness build,
                      oracle/make_harness.py: the configuration's own pulse)
  full_c2_slice_<r>   the 600 x 600 grid (velocity gauge, cos4): the k-block
                      that ParaRange (utility.h:104-115) gives rank r of 160,
                      2 250 k-points, over all 35 303 steps

Each whole-grid case runs as --procs emulated MPI ranks (REF_RANK/REF_SIZE of
oracle/refshim/mpi.h) that dump their partial k-sums at the final reduce
(REF_DUMP); the partial sums are added in rank order, as the reduce
(antelope.cpp:482-512) does, and turned into the columns of the output files
the way antelope.cpp:514-542 writes them (currents times dV, occupations over
Ntotal).  A slice keeps the rank's raw weighted sums.  Stored: the in-plane
current columns (the out-of-plane ones are identically zero for these
pulses) and the occupations; slices also the off-diagonal density matrix sum.

Usage:  python tests/golden/make_golden_full.py [names] [--procs N]
(about 30 minutes of all cores of an 8-core host for all cases).
"""
import concurrent.futures as cf
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from antelope_b200 import workloads  # noqa: E402
from antelope_b200.dist import para_range  # noqa: E402
from oracle import pyoracle  # noqa: E402

SLICE_SIZE = 160        # emulated ranks of the 600 x 600 slices
SLICE_RANKS = (0, 117)  # the first block and one past the middle of the grid


def c1(gauge: str, env: str) -> dict:
    c = workloads.haldane_case(n=150, env=env, gauge=gauge)
    del c["calc"]["precision"]
    return c


def c2() -> dict:
    c = workloads.haldane_case(n=600, env="cos4")
    del c["calc"]["precision"]
    return c


FULL_CASES = {
    "c1_vg_cos4": (c1("Velocity", "cos4"), False),
    "c1_lw_cos4": (c1("Wannier", "cos4"), False),
    "c1_vg_sin2": (c1("Velocity", "sin2"), True),
}
SLICE_CASES = {f"c2_slice_{r}": (c2(), r) for r in SLICE_RANKS}


def run_rank(case, harness, rank, size, workdir):
    prefix = os.path.join(workdir, f"dump_r{rank}")
    pyoracle.run_reference(case, os.path.join(workdir, f"r{rank}"), harness=harness, read=False,
                           env={"REF_RANK": str(rank), "REF_SIZE": str(size), "REF_DUMP": prefix},
                           timeout=24 * 3600)
    return prefix


def whole_grid(name, case, harness, procs):
    d = pyoracle.dims(case)
    Nt, N, nk = d["Nt"], d["nband"], d["ntotal"]
    with tempfile.TemporaryDirectory() as work:
        with cf.ThreadPoolExecutor(procs) as pool:
            prefixes = list(pool.map(lambda r: run_rank(case, harness, r, procs, work), range(procs)))
        inter = np.zeros((Nt, 3))
        intra = np.zeros((Nt, 3))
        dmi = np.zeros((Nt, N, N), dtype=np.complex128)
        for p in prefixes:   # rank order
            s = pyoracle.read_reduce_dumps(p, Nt, N)
            inter += s["inter"]
            intra += s["intra"]
            dmi += s["dmi"]
    occ = np.real(np.einsum("tii->ti", dmi))
    occ_file = np.concatenate([occ / nk, occ.sum(axis=1, keepdims=True) / nk], axis=1)
    np.savez_compressed(os.path.join(HERE, f"full_{name}.npz"),
                        inter=inter[:, :2] * d["dV"], intra=intra[:, :2] * d["dV"], occ_file=occ_file,
                        Nt=Nt, ntotal=nk, procs=procs)
    print(name, Nt, nk, flush=True)


def one_slice(name, case, rank):
    d = pyoracle.dims(case)
    Nt, N, nk = d["Nt"], d["nband"], d["ntotal"]
    kb, ke = para_range(nk, SLICE_SIZE, rank)
    with tempfile.TemporaryDirectory() as work:
        s = pyoracle.read_reduce_dumps(run_rank(case, False, rank, SLICE_SIZE, work), Nt, N)
    np.savez_compressed(os.path.join(HERE, f"full_{name}.npz"),
                        inter=s["inter"][:, :2], intra=s["intra"][:, :2],
                        rho00=s["dmi"][:, 0, 0].real, rho11=s["dmi"][:, 1, 1].real, rho01=s["dmi"][:, 0, 1],
                        k_begin=kb, k_end=ke, size=SLICE_SIZE, rank=rank, Nt=Nt)
    print(name, Nt, kb, ke, flush=True)


def main(argv):
    procs = os.cpu_count() or 1
    if "--procs" in argv:
        i = argv.index("--procs")
        procs = int(argv[i + 1])
        argv = argv[:i] + argv[i + 2:]
    names = argv or list(FULL_CASES) + list(SLICE_CASES)
    with cf.ThreadPoolExecutor(len(SLICE_CASES)) as pool:
        futs = [pool.submit(one_slice, n, *SLICE_CASES[n]) for n in names if n in SLICE_CASES]
        for n in names:
            if n in FULL_CASES:
                whole_grid(n, *FULL_CASES[n], procs)
        for f in futs:
            f.result()


if __name__ == "__main__":
    main(sys.argv[1:])
