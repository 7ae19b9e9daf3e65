"""Small problems on which the reference itself (oracle/_ref) was run to make
the golden fixtures in this folder; also used by the GPU parity tests.

Each case is the dict form of an inputParam.cfg (antelope_b200.cfgtext).
The grids are tiny and the pulses short so that the reference finishes in
about a second per case.
"""
import copy

HALDANE = {"a0": 1.44, "t1": 0.075, "t2": 0.025, "Mt2": 2.54, "phi0": 1.16}

BASE = {
    "target": "Haldane",
    "gauge": "Velocity",
    "laser": {"offset": [0.0, 0.0],
              "pulses": [{"E0": 0.0045, "w0": 0.0855, "ncycles": 2.0, "ellip": 0.0, "cep": 0.0,
                          "t0": 0.0, "phix": 0.0, "env_name": "cos4"}]},
    "calc": {"Npoints": [8, 10], "dt": 0.1, "T1": -1.0, "T2": 220.0, "RKorder": 4,
             "InterIntra": True, "ksfactor": [1.0, 1.0, 1.0]},
    "Haldane": dict(HALDANE),
}


def variant(base=BASE, **kw):
    """Copy ``base`` and set keys given as section__key=value
    (section: top, pulse, laser, calc or the material group)."""
    c = copy.deepcopy(base)
    for k, v in kw.items():
        sect, key = k.split("__")
        if sect == "top":
            c[key] = v
        elif sect == "pulse":
            c["laser"]["pulses"][0][key] = v
        else:
            c[sect][key] = v
    return c


def two_color():
    c = variant(calc__Npoints=[9, 7])
    c["laser"]["pulses"].append({"E0": 0.0015, "w0": 0.171, "ncycles": 4.0, "ellip": 0.0,
                                 "cep": 75.0, "t0": 0.0, "phix": 0.0, "env_name": "cos4"})
    return c


GOLDEN_CASES = {
    "vg_rk4": variant(),
    "vg_rk5_default_order": variant(calc__RKorder=5),
    "lw_rk4": variant(top__gauge="Wannier"),
    "lw_total_current": variant(top__gauge="Wannier", calc__InterIntra=False),
    "vg_total_current": variant(calc__InterIntra=False),
    "lw_t1_elliptic": variant(top__gauge="LengthWannier", calc__T1=300.0, pulse__ellip=0.5,
                              pulse__phix=30.0, pulse__cep=40.0),
    "vg_fermi_t1": variant(Haldane__Ef=0.0, calc__T1=150.0, pulse__ellip=-1.0),
    "vg_cos4_clipped_tilted": variant(pulse__env_name="cos4_clipped", pulse__ncycles_clipped=1.0,
                                      pulse__thetaz=20.0, pulse__phiz=40.0),
    "vg_gauss_clipped_offsets": variant(pulse__env_name="gauss_clipped", pulse__ncycles=0.5,
                                        pulse__ncycles_clipped=1.0, laser__offset=[20.0, 30.0]),
    "vg_gauss_M0_ksfactor": variant(pulse__env_name="gauss", pulse__ncycles=0.7,
                                    Haldane__M0=0.02, calc__ksfactor=[0.5, 0.8, 1.0],
                                    calc__Npoints=[11, 5]),
    "vg_two_color": two_color(),
    "lw_bzaxes_override": variant(top__gauge="Wannier", calc__Npoints=[6, 7],
                                  calc__BZaxes=[1.2, 0.1, 0.0, -0.2, 0.9, 0.0, 0.0, 0.0, 0.0],
                                  calc__BZorigin=[0.05, -0.1]),
    "no_gauge_given_defaults_to_lw": {k: v for k, v in variant(calc__Npoints=[6, 6]).items()
                                      if k != "gauge"},
}

# The reference's other analytic materials (Materials/*.h), run on the GPU as
# Fourier tables of H(k) and of their GenJMatrix (antelope_b200/csrc/
# sbe_materials.cpp); each in both gauges on a small grid.
MATERIALS = {
    "WilsonMass": {"t": 0.02, "delta": 0.015, "mu": -0.03, "a0": 5.0, "a1": 6.0},
    "KaneMele": {"t1": 0.075, "t2": 0.025, "tR": 0.01, "Mt2": 1.5, "phi0": 1.16, "a0": 1.44},
    "Haldane2L": {"t1": 0.075, "t2": 0.025, "phi0": 1.16, "a0": 1.44, "t11": 0.01, "polytype": "AB",
                  "Mt2": 2.0, "t2_bottom": 0.02, "Mt2_bottom": 1.0},
    "XYHlattice": {"tl": 0.05, "tr": 0.03, "lambda": 0.01, "a0": 2.5},
    "TMDCs": {"Material": "MoS2"},
    "SquareSBand": {"t1": 0.02, "M0": 0.03, "a0": 2.0},
    "Bi2Se3surf": {},   # parameters hard-coded in the reference
}


def material(name, gauge, **kw):
    c = variant(top__gauge=gauge, calc__Npoints=[6, 5], **kw)
    del c["Haldane"]
    c["target"] = name
    c[name] = dict(MATERIALS[name])
    return c


MATERIAL_CASES = {f"{m.lower()}_{g[0].lower()}": material(m, g) for m in MATERIALS for g in ("Velocity", "Wannier")}


# MultiWSM (Materials/MultiWSM.h): the continuum two-band model on a 3-D grid
# around k = 0, the parameters of the reference's InputParams/MultiWSM.cfg.
# Its GenJMatrix divides 0 by 0 on the k_x = k_y = 0 line, so the k_x and
# k_y point counts are even (no grid point there).
def multiwsm(gauge, n=1.0, Npoints=(6, 6, 4), **kw):
    c = variant(top__gauge=gauge, calc__Npoints=list(Npoints), pulse__ellip=0.3, **kw)
    del c["Haldane"]
    c["target"] = "MultiWSM"
    c["MultiWSM"] = {"n": float(n), "v": 0.2, "alphan": 0.1, "phi0": 0.1, "a0": 1.0}
    return c


MULTIWSM_CASES = {
    "multiwsm_v": multiwsm("Velocity"),
    "multiwsm_w": multiwsm("Wannier"),
    "multiwsm_w_n2_tilted": multiwsm("Wannier", n=2.0, Npoints=(4, 4, 4), pulse__thetaz=30.0, pulse__phiz=20.0),
}
# Bi2Se3surf's bands meet where every sin(k.a_i) vanishes, e.g. at
# (pi/a0, pi/(sqrt(3) a0)), a grid point whenever Npoints[1] - 1 is a multiple
# of 4; per-band quantities there depend on the eigensolver's basis, so its
# cases use a 6 x 6 grid, which avoids those points.
for _g in ("v", "w"):
    MATERIAL_CASES[f"bi2se3surf_{_g}"]["calc"]["Npoints"] = [6, 6]
# reference specifics exercised on purpose: WilsonMass without a1 (a1 = a0);
# Haldane2L stackings with a flipped B2 sign and t1_bottom read first (the
# OR short-circuit leaves t2_bottom unread); Kane-Mele with T1 and no Rashba
_h2l = material("Haldane2L", "Wannier", calc__T1=300.0)
_h2l["Haldane2L"].update(polytype="AA'", t1_bottom=0.07, t2_bottom=0.03)
_wm = material("WilsonMass", "Velocity", pulse__ellip=0.4)
del _wm["WilsonMass"]["a1"]
_km = material("KaneMele", "Velocity", calc__T1=150.0)
_km["KaneMele"]["tR"] = 0.0
_h2lv = material("Haldane2L", "Velocity")
_h2lv["Haldane2L"].update(polytype="A'B", M0=0.01)
_soc = {g: material("TMDCs", g) for g in ("Velocity", "Wannier")}
for g, c in _soc.items():
    c["TMDCs"] = {"Material": "WSe2", "isSOCEnabled": True}
MATERIAL_CASES.update({"haldane2l_w_2h_t1bottom": _h2l, "wilsonmass_v_default_a1": _wm,
                       "kanemele_v_t1_no_rashba": _km, "haldane2l_v_apb_m0": _h2lv,
                       "tmdcs_v_wse2_soc": _soc["Velocity"], "tmdcs_w_wse2_soc": _soc["Wannier"]})

# Bands degenerate at grid points: per-band values there depend on the basis
# chosen inside the degenerate subspace (LAPACK zheevr's in the reference,
# unpinned; a rounding-level change of H(k) changes the Jacobi solvers'
# choice), so band-basis occupations are compared summed over each group.
# Kane-Mele without Rashba: two uncoupled Haldane blocks (phi0, -phi0) whose
# valence bands coincide on the ky = 0 row; WSe2 with spin-orbit coupling:
# spin pairs meet where the splitting vanishes.
BAND_GROUPS = {"kanemele_v_t1_no_rashba": [[0, 1], [2, 3]],
               "tmdcs_v_wse2_soc": [[0, 1], [2, 3], [4, 5]]}

# Density snapshots (calc.shotNumber, antelope.cpp:267-422): the 1-D integrated
# conduction occupation and the per-k conduction occupation and coherence
# every int(period0 / shotNumber / dt) steps.
_km_shots = material("KaneMele", "Wannier", calc__shotNumber=2)
SNAPSHOT_CASES = {
    "vg_shots": variant(calc__shotNumber=4),
    "lw_shots": variant(top__gauge="Wannier", calc__shotNumber=3, calc__Npoints=[7, 6]),
    "vg_shots_fermi_t1": variant(Haldane__Ef=0.0, calc__T1=150.0, calc__shotNumber=5, pulse__ellip=0.3),
    "kanemele_w_shots": _km_shots,
    "tmdcs_v_shots": material("TMDCs", "Velocity", calc__shotNumber=3),
}

# A one-cycle case whose output files are kept verbatim (byte format pin).
TEXT_CASE = variant(pulse__ncycles=1.0, pulse__w0=0.114, calc__Npoints=[5, 6])

# Cases the harness build of the reference runs (oracle/make_harness.py: its
# SBEs.h and laser.h with the sin2 envelope and the SyntheticWannier material
# of oracle/refharness/SyntheticWannier.h, which has dipole matrices).  They pin
# what the unmodified reference cannot run: the sin2 pulse of the
# configurations, the length gauge's E(t).D(k+A) term (SBEs.h:771-782) and the
# current operator -dH/dk + i[D, H] (BaseMaterial.h:62-68) of an N-band model.
def synthetic(gauge, rk=4, seed=4, nband=6, nval=3, npoints=(5, 4), w0=0.057, dipoles=True, **kw):
    from antelope_b200 import wannier

    c = variant(top__gauge=gauge, calc__Npoints=list(npoints), calc__RKorder=rk, pulse__w0=w0,
                pulse__ncycles=0.5, pulse__env_name="sin2", **kw)
    del c["Haldane"]
    c["target"] = "SyntheticWannier"
    g = wannier.generate(seed, nband=nband, nval=nval)
    if not dipoles:
        del g["d_re"], g["d_im"]
    c["SyntheticWannier"] = g
    return c


HARNESS_CASES = {
    "sin2_vg_rk4": variant(pulse__env_name="sin2"),
    "sin2_lw_rk5_elliptic": variant(top__gauge="Wannier", pulse__env_name="sin2", calc__RKorder=5,
                                    pulse__ellip=0.3, pulse__cep=25.0),
    "synw6_w_rk4": synthetic("Wannier", 4),
    "synw6_w_rk5": synthetic("Wannier", 5),
    "synw6_v_rk4": synthetic("Velocity", 4),
    "synw6_v_rk5": synthetic("Velocity", 5),
    "synw6_w_rk4_no_dipoles": synthetic("Wannier", 4, dipoles=False),
    "synw4_w_t1_elliptic": synthetic("Wannier", 4, seed=9, nband=4, nval=2, npoints=(6, 5),
                                     calc__T1=300.0, pulse__ellip=0.5, pulse__phix=20.0),
}
# The N = 6 length-gauge case with the reference's fixed-step Fehlberg-5 at
# dt = 0.025: a fine solution of the same equations by the reference's own
# integrator, against which the adaptive Cash-Karp extension (no counterpart
# in the reference) is shown to converge.
HARNESS_CASES["synw6_w_rk5_fine"] = synthetic("Wannier", 5, calc__dt=0.025)
