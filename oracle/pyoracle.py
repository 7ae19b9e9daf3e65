"""ctypes front end of the C oracle (oracle/sbe_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker, and by bench.py's CPU-baseline leg.  The product package never
imports it.

A *case* is the dict form of an ``inputParam.cfg`` (see
``antelope_b200.cfgtext``): top-level ``target``/``gauge``, a ``laser`` group,
a ``calc`` group and one material group.  ``to_problem`` turns it into the
oracle's ``orc_problem`` struct with the reference's defaults
(SBEs.h:432-509, antelope.cpp:111-129).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_sbe.so")
REF_EXE = os.path.join(HERE, "_ref", "exec_hhg_ref")
# the reference build with the harness additions of make_harness.py (the sin2
# envelope and the SyntheticWannier material with dipoles)
HARNESS_EXE = os.path.join(HERE, "_ref", "exec_hhg_harness")

ENV = {"gauss": 0, "gauss_clipped": 1, "cos4": 2, "cos4_clipped": 3, "sin2": 4}
GAUGE = {"Wannier": 0, "LengthWannier": 0, "Hamiltonian": 1, "LengthHamiltonian": 1,
         "Velocity": 2, "VelocityHamiltonian": 2}
MAX_PULSES = 8


class OrcPulse(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "E0", "w0", "ellip", "ncycles", "cep_deg", "t0", "phix_deg", "ncycles_clipped",
        "thetaz_deg", "phiz_deg")] + [("env", C.c_int)]


class OrcProblem(C.Structure):
    _fields_ = [
        ("npulses", C.c_int), ("pulses", OrcPulse * MAX_PULSES),
        ("offset_before", C.c_double), ("offset_after", C.c_double),
        ("dt", C.c_double), ("T1", C.c_double), ("T2", C.c_double),
        ("rk", C.c_int), ("rk_tol", C.c_double), ("inter_intra", C.c_int), ("gauge", C.c_int),
        ("Nk", C.c_int * 3), ("ksfactor", C.c_double * 3),
        ("n_bzaxes", C.c_int), ("bzaxes", C.c_double * 9),
        ("n_bzorigin", C.c_int), ("bzorigin", C.c_double * 3),
        ("model", C.c_int),
        ("hal_a0_ang", C.c_double), ("hal_t1", C.c_double), ("hal_t2", C.c_double),
        ("hal_M0", C.c_double), ("hal_phi0", C.c_double),
        ("use_fermi", C.c_int), ("Ef", C.c_double),
        ("w_nband", C.c_int), ("w_nval", C.c_int), ("w_nR", C.c_int),
        ("w_R", C.POINTER(C.c_int)), ("w_lat", C.c_double * 4),
        ("w_h", C.POINTER(C.c_double)), ("w_d", C.POINTER(C.c_double)),
        ("w_vec", C.POINTER(C.c_double)), ("w_j", C.POINTER(C.c_double)), ("w_bz", C.c_double * 9),
        ("nthreads", C.c_int),
        ("mw_n", C.c_double), ("mw_v", C.c_double), ("mw_alphan", C.c_double), ("mw_a0_ang", C.c_double),
    ]


class OrcDims(C.Structure):
    _fields_ = [("Nt", C.c_int), ("nband", C.c_int), ("nval", C.c_int), ("ntotal", C.c_int),
                ("atmin", C.c_double), ("dV", C.c_double), ("total_weight", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE, "port"])
        _lib = C.CDLL(LIB_PATH)
        _lib.orc_get_dims.argtypes = [C.POINTER(OrcProblem), C.POINTER(OrcDims)]
        _lib.orc_run.argtypes = [C.POINTER(OrcProblem), C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.POINTER(C.c_long)]
        _lib.orc_run_shots.argtypes = [C.POINTER(OrcProblem), C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(C.c_long), C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_shot_dims.argtypes = [C.POINTER(OrcProblem), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        _lib.orc_laser_eval.argtypes = [C.POINTER(OrcProblem), C.c_double, C.c_void_p, C.c_void_p]
        _lib.orc_kgrid.argtypes = [C.POINTER(OrcProblem), C.c_void_p, C.c_void_p]
        _lib.orc_model_hj.argtypes = [C.POINTER(OrcProblem), C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_eigh.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_tableau.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


MATERIAL_TABLES = ("KaneMele", "Haldane2L", "WilsonMass", "XYHlattice", "TMDCs", "SquareSBand", "Bi2Se3surf")


def to_problem(case: dict, nthreads: int = 1):
    """Build an ``orc_problem`` (and the arrays it points to) from a case dict."""
    p = OrcProblem()
    keep = []
    laser = case["laser"]
    pulses = laser["pulses"]
    if not 1 <= len(pulses) <= MAX_PULSES:
        raise ValueError("1..8 pulses supported")
    p.npulses = len(pulses)
    for i, q in enumerate(pulses):
        o = p.pulses[i]
        o.E0, o.w0, o.ellip, o.ncycles = q["E0"], q["w0"], q["ellip"], q["ncycles"]
        o.cep_deg, o.t0, o.phix_deg = q["cep"], q["t0"], q["phix"]
        o.ncycles_clipped = q.get("ncycles_clipped", 0.0)
        o.thetaz_deg, o.phiz_deg = q.get("thetaz", 0.0), q.get("phiz", 0.0)
        o.env = ENV[q["env_name"]]
    off = laser.get("offset", [0.0, 0.0])
    p.offset_before, p.offset_after = off[0], off[1]
    calc = case["calc"]
    p.dt = calc.get("dt", 0.1)
    p.T1 = calc.get("T1", -1.0)
    p.T2 = calc.get("T2", -1.0)
    rk = calc.get("rk", None)   # extension key; overrides RKorder when present
    p.rk = {"rk4": 4, "rk5": 5, "fehlberg5": 5, "cashkarp45": 45}[rk] if rk else int(calc.get("RKorder", 5))
    p.rk_tol = calc.get("tol", 1e-8)
    p.inter_intra = 1 if calc.get("InterIntra", False) else 0
    p.gauge = GAUGE.get(case.get("gauge", ""), 0)
    npts = list(calc["Npoints"]) + [1] * (3 - len(calc["Npoints"]))
    for i in range(3):
        p.Nk[i] = npts[i]
    ks = list(calc["ksfactor"]) + [1.0] * (3 - len(calc["ksfactor"]))
    for i in range(3):
        p.ksfactor[i] = ks[i]
    if "BZaxes" in calc:
        p.n_bzaxes = len(calc["BZaxes"])
        for i, v in enumerate(calc["BZaxes"]):
            p.bzaxes[i] = v
    if "BZorigin" in calc:
        p.n_bzorigin = len(calc["BZorigin"])
        for i, v in enumerate(calc["BZorigin"]):
            p.bzorigin[i] = v
    target = case["target"]
    mat = case.get(target, {})
    if "Ef" in mat:
        p.use_fermi, p.Ef = 1, mat["Ef"]
    if target == "Haldane":
        p.model = 0
        p.hal_a0_ang, p.hal_t1, p.hal_t2, p.hal_phi0 = mat["a0"], mat["t1"], mat["t2"], mat["phi0"]
        p.hal_M0 = mat["M0"] if "M0" in mat else mat["Mt2"] * mat["t2"]
    elif target == "MultiWSM":
        # the continuum two-band model (Materials/MultiWSM.h), restated in C
        p.model = 2
        p.mw_n, p.mw_v, p.mw_alphan, p.mw_a0_ang = mat["n"], mat["v"], mat["alphan"], mat["a0"]
    elif target == "SyntheticWannier":
        # explicit tight-binding tables of the cfg group (Nband, Nval, lattice,
        # R pairs, h_re/h_im [nR][N][N], optional d_re/d_im [nR][2][N][N])
        N = int(mat["Nband"])
        R = np.ascontiguousarray(np.asarray(mat["R"], dtype=np.int32).reshape(-1, 2))
        nR = len(R)
        h = np.ascontiguousarray((np.asarray(mat["h_re"]) + 1j * np.asarray(mat["h_im"])).reshape(nR, N, N))
        keep += [R, h]
        p.model = 1
        p.w_nband, p.w_nval, p.w_nR = N, int(mat["Nval"]), nR
        p.w_R = R.ctypes.data_as(C.POINTER(C.c_int))
        p.w_h = h.ctypes.data_as(C.POINTER(C.c_double))
        if "d_re" in mat:
            d = np.ascontiguousarray((np.asarray(mat["d_re"]) + 1j * np.asarray(mat["d_im"])).reshape(nR, 2, N, N))
            keep.append(d)
            p.w_d = d.ctypes.data_as(C.POINTER(C.c_double))
        for i, v in enumerate(mat["lattice"]):
            p.w_lat[i] = float(v)
    elif target in MATERIAL_TABLES:
        # an analytic material (Materials/*.h): its H and GenJMatrix as Fourier
        # tables, read from the product's cfg front end (sbe_problem_model).
        # The tables are checked end to end against the reference's own runs
        # of the same cfgs (tests/golden), so the oracle's engine and the
        # restated material are pinned together.
        from antelope_b200 import Problem
        t = Problem.from_dict(case).model_tables()
        N, nR = t["nband"], len(t["vec"])
        vec = np.ascontiguousarray(t["vec"])
        h = np.ascontiguousarray(t["h"])
        j = np.ascontiguousarray(t["j"])
        keep += [vec, h, j]
        p.model = 1
        p.w_nband, p.w_nval, p.w_nR = N, t["nval"], nR
        p.w_vec = vec.ctypes.data_as(C.POINTER(C.c_double))
        p.w_h = h.ctypes.data_as(C.POINTER(C.c_double))
        p.w_j = j.ctypes.data_as(C.POINTER(C.c_double))
        for i in range(9):
            p.w_bz[i] = t["bz"][i]
    else:
        raise ValueError(f"oracle has no model '{target}'")
    p.nthreads = nthreads
    p._keep = keep
    return p


def dims(case: dict) -> dict:
    p = to_problem(case)
    d = OrcDims()
    if lib().orc_get_dims(C.byref(p), C.byref(d)) != 0:
        raise ValueError("oracle rejected the case")
    return {f: getattr(d, f) for f, _ in OrcDims._fields_}


def shot_dims(case: dict):
    """(interval F, number of snapshots) for the case's calc.shotNumber."""
    p = to_problem(case)
    every, n = C.c_int(0), C.c_int(0)
    rc = lib().orc_shot_dims(C.byref(p), int(case["calc"].get("shotNumber", 0)), C.byref(every), C.byref(n))
    if rc != 0:
        raise ValueError(f"no snapshot interval for this case ({rc})")
    return every.value, n.value


def run(case: dict, nthreads: int = 1) -> dict:
    """Propagate a case on the CPU.  Returns the arrays the reference writes:
    ``inter``/``intra`` [Nt,3] (already times dV), ``occ`` [Nt,N] and the raw
    weighted density-matrix integral ``dmi`` [Nt,N,N] (complex).  With
    calc.shotNumber > 0 also the snapshots: ``occ1d`` [nshots,N0] and the
    per-k ``nc`` [nshots,Ntotal] and ``pi`` [nshots,Ntotal] (complex)."""
    p = to_problem(case, nthreads)
    d = dims(case)
    Nt, N = d["Nt"], d["nband"]
    inter = np.zeros((Nt, 3))
    intra = np.zeros((Nt, 3))
    dmi = np.zeros((Nt, N, N), dtype=np.complex128)
    steps = C.c_long(0)
    shots = int(case["calc"].get("shotNumber", 0))
    out = {}
    if shots > 0:
        _, ns = shot_dims(case)
        n0 = int(case["calc"]["Npoints"][0])
        occ1d = np.zeros((ns, n0))
        nc = np.zeros((ns, d["ntotal"]))
        pi = np.zeros((ns, d["ntotal"]), dtype=np.complex128)
        rc = lib().orc_run_shots(C.byref(p), shots, _ptr(inter), _ptr(intra), _ptr(dmi), C.byref(steps),
                                 _ptr(occ1d), _ptr(nc), _ptr(pi))
        out = {"occ1d": occ1d, "nc": nc, "pi": pi}
    else:
        rc = lib().orc_run(C.byref(p), _ptr(inter), _ptr(intra), _ptr(dmi), C.byref(steps))
    if rc != 0:
        raise RuntimeError(f"oracle run failed ({rc})")
    occ = np.real(np.einsum("tii->ti", dmi)) / d["ntotal"]
    return {"inter": inter, "intra": intra, "dmi": dmi, "occ": occ, "dims": d,
            "steps": steps.value, **out}


def laser_eval(case: dict, t: float):
    p = to_problem(case)
    A = np.zeros(3)
    E = np.zeros(3)
    lib().orc_laser_eval(C.byref(p), float(t), _ptr(A), _ptr(E))
    return A, E


def kgrid(case: dict):
    p = to_problem(case)
    n = dims(case)["ntotal"]
    k = np.zeros((n, 3))
    w = np.zeros(n)
    lib().orc_kgrid(C.byref(p), _ptr(k), _ptr(w))
    return k, w


def model_hj(case: dict, k3):
    p = to_problem(case)
    N = dims(case)["nband"]
    H = np.zeros((N, N), dtype=np.complex128)
    J = np.zeros((3, N, N), dtype=np.complex128)
    k = np.ascontiguousarray(k3, dtype=np.float64)
    lib().orc_model_hj(C.byref(p), _ptr(k), _ptr(H), _ptr(J))
    return H, J


def eigh(a):
    a = np.ascontiguousarray(a, dtype=np.complex128)
    n = a.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n), dtype=np.complex128)
    if lib().orc_eigh(n, _ptr(a), _ptr(w), _ptr(v)) != 0:
        raise ValueError("bad size")
    return w, v


def tableau(rk: int):
    """(c, a, b, bstar) of the oracle's integrator for rk = 4, 5 or 45."""
    c, b, bs = np.zeros(7), np.zeros(7), np.zeros(7)
    a = np.zeros((7, 7))
    s = lib().orc_tableau(int(rk), _ptr(c), _ptr(a), _ptr(b), _ptr(bs))
    if s < 0:
        raise ValueError(f"no tableau for rk={rk}")
    return c[:s], a[:s, :s], b[:s], bs[:s]


def run_reference(case: dict, workdir: str, env: dict | None = None, timeout: float = 3600,
                  harness: bool = False, read: bool = True):
    """Run the unmodified reference build (oracle/_ref/exec_hhg_ref) -- or,
    with ``harness``, the harness build with the sin2 envelope and the
    SyntheticWannier material -- on a case in ``workdir``; returns the parsed
    output files (``read``)."""
    from antelope_b200 import cfgtext

    exe = HARNESS_EXE if harness else REF_EXE
    if not os.path.exists(exe):
        raise FileNotFoundError(f"{exe} not built (needs the reference sources)")
    os.makedirs(workdir, exist_ok=True)
    with open(os.path.join(workdir, "inputParam.cfg"), "w") as f:
        f.write(cfgtext.dumps(case))
    e = dict(os.environ)
    if env:
        e.update(env)
    subprocess.run([exe], cwd=workdir, env=e, check=True, timeout=timeout,
                   stdout=subprocess.DEVNULL)
    return read_outputs(workdir) if read else None


def read_reduce_dumps(prefix: str, Nt: int, N: int) -> dict:
    """The partial k-sums one emulated rank dumped at the reference's final
    reduce (REF_DUMP, oracle/refshim/mpi.h; antelope.cpp:482-512): inter and
    intra [Nt, 3] (weighted, before the factor dV) and the weighted density
    matrix ``dmi`` [Nt, N, N].  Snapshot reduces, if any, come first."""
    import glob

    files = sorted(glob.glob(prefix + ".*.bin"), key=lambda f: int(f.rsplit(".", 2)[1]))
    tail = files[-7:]
    arr = [np.fromfile(f, dtype=np.complex128) for f in tail]
    inter = np.stack([arr[0], arr[2], arr[4]], axis=1).real
    intra = np.stack([arr[1], arr[3], arr[5]], axis=1).real
    dmi = arr[6].reshape(Nt, N, N)
    return {"inter": inter, "intra": intra, "dmi": dmi}


def read_outputs(workdir: str) -> dict:
    """The reference's output files as arrays; the snapshot files
    (antelope.cpp:288-292, 416-421) when they exist: ``occ1d`` [nshots,N0]
    (text), ``nc`` (binary doubles) and ``pi`` (binary complex doubles) as flat
    arrays of nshots * Ntotal values."""
    def load(name):
        return np.loadtxt(os.path.join(workdir, name), ndmin=2)

    out = {"inter": load("interband_dipole_full_evol.dat"),
           "intra": load("intraband_current_full_evol.dat"),
           "occ_file": load("occupation__full__evol.dat"),
           "coh_file": load("coherence__full__evol.dat"),
           "laser": load("outlaserdata.dat")}
    if os.path.exists(os.path.join(workdir, "occupation_1d_integration.dat")):
        out["occ1d"] = load("occupation_1d_integration.dat")
        out["nc"] = np.fromfile(os.path.join(workdir, "fisrt_conduction.dat"), dtype=np.float64)
        out["pi"] = np.fromfile(os.path.join(workdir, "fisrt_coherence.dat"), dtype=np.complex128)
    return out
