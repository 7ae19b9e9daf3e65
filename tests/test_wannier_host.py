"""SyntheticWannier input handling (no GPU): the cfg tables round-trip, the
grid/time axis agree with the oracle, and malformed models are refused."""
import copy

import numpy as np
import pytest

import antelope_b200 as ab
from antelope_b200 import wannier
from antelope_b200.api import SbeError
from oracle import pyoracle


def test_generator_is_hermitian_and_seeded():
    g = wannier.generate(7)
    m = wannier.synthetic_model(g)
    R = [tuple(r) for r in m["R"]]
    assert len(R) == 37 and (0, 0) in R
    for i, r in enumerate(R):
        j = R.index((-r[0], -r[1]))
        assert np.allclose(m["h"][j], m["h"][i].conj().T)
        assert np.allclose(m["d"][j], np.conj(np.swapaxes(m["d"][i], 1, 2)))
    assert wannier.generate(7) == g and wannier.generate(8) != g


def test_dims_match_oracle():
    c = wannier.wannier_case(seed=2, n=9, ncycles=1.0)
    p = ab.Problem.from_dict(c)
    d = pyoracle.dims(c)
    assert (p.dims.Nt, p.dims.nband, p.dims.nval, p.dims.ntotal) == (d["Nt"], 6, 3, 81)
    assert p.dims.dV == d["dV"] and p.dims.atmin == d["atmin"] and p.dims.rk == 45


def test_rejects_non_hermitian_model():
    c = wannier.wannier_case(seed=2, n=9, ncycles=1.0)
    c["SyntheticWannier"]["h_im"][5] += 0.01
    with pytest.raises(SbeError) as e:
        ab.Problem.from_dict(c)
    assert e.value.name == "SBE_BAD_CONFIG" and "dagger" in str(e.value)


def test_velocity_gauge_wannier_parses():
    """Wannier models also run in the velocity gauge (band basis of H(k),
    P = U^dag J U with J = -dH/dk + i[D, H]); the dims follow the tables."""
    c = wannier.wannier_case(seed=2, n=9, ncycles=1.0, gauge="Velocity")
    p = ab.Problem.from_dict(c)
    assert p.dims.nband == 6 and p.dims.gauge == 2
    t = p.model_tables()
    assert t["d"] is not None and t["j"] is None
