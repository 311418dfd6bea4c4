"""C-ABI library: exports, host-only set-up parity and error behaviour (CPU).

The host set-up of wfe_b200 (config parsing, Gal-Chen metric, hydrostatic base
state, initial conditions) runs without a GPU when a context is created with
device = -1; its FP64 arrays must be bit-identical to the reference's FP64
build (golden vectors) and to the CPU oracle.
"""

import re

import numpy as np
import pytest

import oracle as O
import wfe_b200 as W
from helpers import CASES, ROOT, golden

RUN_CASES = ["bubble_open", "straka_periodic", "schaer_open", "wk82_small", "moist_blob",
             "ops_open", "ops_periodic"]


def header_symbols():
    text = (ROOT / "include" / "wfe_b200.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|long|const char\*|void\*)\s+(wfe_\w+)\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = W.load_library()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(W.SYMBOLS) == syms


@pytest.mark.parametrize("case", RUN_CASES)
def test_host_setup_bit_identical_to_reference(case):
    G = golden(case)
    c = W.Case(CASES / f"{case}.ini", precision="f64", device=-1)
    for k in W.METRIC:
        assert np.array_equal(c.metric(k), G["m_" + k]), k
    for k in W.BASE:
        assert np.array_equal(c.base(k), G["b_" + k], equal_nan=True), k
    o = O.Case(CASES / f"{case}.ini")
    assert (c.nx, c.ny, c.nz, c.NX, c.NY, c.NZ) == (o.grid.nx, o.grid.ny, o.grid.nz, o.grid.NX,
                                                   o.grid.NY, o.grid.NZ)
    assert c.moisture == o.params.moisture and c.pd_moist == o.params.pd_moist
    assert c.zt == o.zt


def test_host_only_context_refuses_device_work():
    c = W.Case(CASES / "bubble_open.ini", device=-1)
    with pytest.raises(W.WfeError) as e:
        c.step()
    assert e.value.code == 2
    with pytest.raises(W.WfeError):
        c.field("u")


def test_config_errors():
    with pytest.raises(W.WfeError) as e:
        W.Case(CASES / "no_such_case.ini", device=-1)
    assert e.value.code == 3
    with pytest.raises(W.WfeError) as e:
        W.Case(CASES / "bubble_open.ini", {"profile": "nonsense"}, device=-1)
    assert e.value.code == 3 and "unknown profile" in str(e.value)
    with pytest.raises(W.WfeError) as e:
        W.Case(CASES / "bubble_open.ini", {"profile": "file", "input_dir": "/nonexistent"},
               device=-1)
    assert e.value.code == 4
    with pytest.raises(W.WfeError) as e:
        W.Case(CASES / "bubble_open.ini", {"nz": 2}, device=-1)
    assert e.value.code == 3


def test_overrides_and_text_create():
    text = (CASES / "bubble_open.ini").read_text()
    a = W.Case(text=text, overrides={"nx": 20, "wind_profile": "linear", "wind_us": 35,
                                     "wind_zs": 1500}, device=-1)
    assert a.nx == 20
    ub = a.base("ub")
    o = O.Case(CASES / "bubble_open.ini", {"nx": 20, "wind_profile": "linear", "wind_us": 35,
                                           "wind_zs": 1500})
    assert np.array_equal(ub, o.base["ub"])
    zc = a.metric("zeta_c")[3:3 + a.nz]
    expect = np.minimum(np.maximum(zc, 0) / 1500.0, 1.0) * 35
    assert np.allclose(ub[3:3 + a.nz], expect, rtol=0, atol=1e-12)
