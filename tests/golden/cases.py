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

# A one-cycle case whose output files are kept verbatim (byte format pin).
TEXT_CASE = variant(pulse__ncycles=1.0, pulse__w0=0.114, calc__Npoints=[5, 6])
