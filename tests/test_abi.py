"""CPU checks of the C-ABI library: it loads without a GPU and exports every entry point that
include/neon_b200.h declares; the host-side restatements (problem set-up) behave like neon."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from neon_b200 import problem as P


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for h in os.listdir(inc):
        if h.endswith(".h"):
            src = open(os.path.join(inc, h)).read()
            names |= set(re.findall(r"^int (nb2_\w+)\(", src, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    assert "nb2_create" in names and "nb2_static_solve" in names and "nb2_pcg_solve" in names


def test_library_exports_every_declared_symbol():
    from neon_b200 import api
    if not os.path.exists(api.LIB_PATH):
        from neon_b200 import build
        build.build()
    L = ctypes.CDLL(api.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(L, n)]
    assert not missing, missing
    # the Python mirror binds every declared symbol too
    assert set(_declared()) <= set(api._SIGS)


def test_create_rejects_bad_input_without_gpu():
    from neon_b200 import api
    L = api.lib()
    X = np.zeros((4, 3))
    conn = np.array([[0, 1, 2, 7]], np.int32)  # node 7 does not exist
    desc = api.MeshDesc(4, X.ctypes.data, 1, 4, conn.ctypes.data)
    mat = api.MaterialDesc(0, 1.0, 1.0, 0, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    assert L.nb2_create(ctypes.byref(desc), ctypes.byref(mat), ctypes.byref(h)) == api.E_INPUT
    buf = ctypes.create_string_buffer(256)
    L.nb2_last_error(None, buf, 256)
    assert b"connectivity" in buf.value


def test_material_factory_semantics():
    m = P.make_material({"elastic_modulus": 200e3, "poissons_ratio": 0.3},
                        {"name": "isotropic_linear_elasticity"})
    assert m.K == pytest.approx(200e3 / (3 * 0.4)) and m.G == pytest.approx(200e3 / 2.6)
    with pytest.raises(ValueError):
        P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.5}, {"name": "neohooke"})
    with pytest.raises(ValueError):
        P.make_material({"elastic_modulus": 1.0, "poissons_ratio": 0.3}, {"name": "J2_plasticity"})
    with pytest.raises(ValueError):
        P.make_material({"shear_modulus": 1.0, "bulk_modulus": 1.0}, {"name": "unknown"})


def test_microsphere_factory_errors():
    """test/hyperelastic_constitutive.cpp "microsphere model error test" and the statistics
    checks of constitutive_model_factory.cpp:48-120."""
    ms = {"name": "microsphere"}
    for constitutive in ({**ms, "Tyasdpe": "affine"}, {**ms, "type": "Afwsfine"},
                         {**ms, "type": "affine", "statistics": "gaussian"},
                         {**ms, "type": "Afwsfine", "quadrature": "BO21"},
                         {**ms, "type": "affine", "quadrature": "BO99"},
                         {**ms, "type": "affine", "quadrature": "BO21"},
                         {**ms, "type": "affine", "quadrature": "BO21", "statistics": "debye"}):
        with pytest.raises(ValueError):
            P.make_material({}, constitutive)
    rubber = {"elastic_modulus": 10e6, "poissons_ratio": 0.45, "segments_per_chain": 50}
    with pytest.raises(ValueError):  # segments_per_chain missing
        P.make_material({"elastic_modulus": 10e6, "poissons_ratio": 0.45},
                        {**ms, "type": "affine", "quadrature": "BO21", "statistics": "langevin"})
    for statistics, model in (("gaussian", P.GAUSS_AFFINE_MICROSPHERE),
                              ("langevin", P.LANGEVIN_AFFINE_MICROSPHERE)):
        m = P.make_material(rubber, {**ms, "type": "affine", "quadrature": "BO21",
                                     "statistics": statistics})
        assert m.model == model and m.segments_per_chain == 50
    with pytest.raises(NotImplementedError):  # the 900-point rule is not on this path
        P.make_material(rubber, {**ms, "type": "affine", "quadrature": "FM900",
                                 "statistics": "langevin"})
    assert P.make_material(rubber, {**ms, "type": "affine", "quadrature": "BO33",
                                    "statistics": "langevin"}).unit_sphere_points == 33
    # test/hyperelastic_constitutive.cpp "Nonaffine microsphere" exception: a misspelt
    # nonaffine_stretch_parameter
    with pytest.raises(ValueError):
        P.make_material({**rubber, "nonaffine_Strearameter": 1.0},
                        {**ms, "type": "nonaffine", "quadrature": "BO21"})
    m = P.make_material({**rubber, "nonaffine_stretch_parameter": 1.0},
                        {**ms, "type": "nonaffine", "quadrature": "BO21"})
    assert m.model == P.NONAFFINE_MICROSPHERE and m.nonaffine_stretch_parameter == 1.0


def test_dirichlet_order_and_sinusoid():
    from neon_b200 import mesh as M
    m = M.structured_hex8(2)
    b = P.dirichlet_boundaries(m, [
        {"name": "top", "time": [0, 1], "z": [0, 1]},
        {"name": "bottom", "time": [0, 1], "x": [0, 0], "z": [0, 0]}])
    assert [(t.name, int(t.dofs[0] % 3)) for t in b] == [("bottom", 0), ("bottom", 2),
                                                         ("top", 2)]
    t, v = P.sinusoidal_table(5e-3, 20.0, 1.0, 0.0, 1.0)
    assert len(t) == 21 and t[0] == 0 and t[-1] == pytest.approx(20.0)
    assert v[5] == pytest.approx(5e-3) and v[15] == pytest.approx(-5e-3)
