"""CPU tests of the C ABI boundary: the library loads, exports every symbol
declared in include/p3mx.h, and validates actor parameters with the
reference's messages (p3m_tuning_exceptions.py:192-225) without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from espresso_b200 import _lib
from espresso_b200.electrostatics import P3M, P3MGPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "p3mx.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(p3mx_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(_lib.SIGNATURES), "ctypes signatures out of sync with the header"
    assert lib.p3mx_version().startswith(b"p3mx")


VALID = {'prefactor': 2.0, 'accuracy': .01, 'tune': False, 'cao': 3, 'r_cut': 0.373,
         'alpha': 3.81, 'mesh': (8, 8, 8), 'epsilon': 0., 'mesh_off': [0.5, 0.5, 0.5]}

INVALID = [
    ('prefactor', -2.0, "Parameter 'prefactor' must be > 0"),
    ('epsilon', -1.0, "Parameter 'epsilon' must be >= 0"),
    ('cao', 0, "Parameter 'cao' must be >= 1 and <= 7"),
    ('cao', 8, "Parameter 'cao' must be >= 1 and <= 7"),
    ('r_cut', -2.0, "Parameter 'r_cut' must be > 0"),
    ('alpha', -2.0, "Parameter 'alpha' must be > 0"),
    ('accuracy', -2.0, "Parameter 'accuracy' must be > 0"),
    ('mesh', (-1, -1, -1), "Parameter 'mesh' must be > 0"),
    ('mesh', (2, 2, 2), "Parameter 'cao' cannot be larger than 'mesh'"),
    ('mesh_off', (-2, 1, 1), "Parameter 'mesh_off' must be >= 0 and <= 1"),
]


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
@pytest.mark.parametrize("key,value,msg", INVALID)
def test_invalid_params(cls, key, value, msg):
    params = dict(VALID)
    params[key] = value
    with pytest.raises(ValueError, match=re.escape(msg)):
        cls(**params)


def test_python_side_validation():
    with pytest.raises(ValueError, match="even number of mesh points"):
        P3M(prefactor=1., accuracy=1e-3, mesh=[7, 8, 8])
    with pytest.raises(TypeError, match="'tune' has to be a boolean"):
        P3M(prefactor=1., accuracy=1e-3, tune=1)
    with pytest.raises(TypeError, match="'timings' has to be an integer"):
        P3M(prefactor=1., accuracy=1e-3, timings=1.5)
    with pytest.raises(ValueError, match="accuracy"):
        P3M(prefactor=1.)


def test_defaults_and_precision():
    a = P3M(prefactor=1., accuracy=1e-3)
    b = P3MGPU(prefactor=1., accuracy=1e-3)
    assert a.single_precision is False and b.single_precision is True
    assert a.timings == 10 and a.tune is True and a.epsilon == 0.0
    assert a.get_params()["mesh"] == [-1, -1, -1]
    assert a.get_params()["mesh_off"] == [0.5, 0.5, 0.5]
    assert a.get_params()["is_tuned"] is False
    c = P3M(prefactor=1., accuracy=1e-3, mesh=16, epsilon="metallic")
    assert c.get_params()["mesh"] == [16, 16, 16]


def test_periodicity_and_state_errors_need_no_gpu():
    lib = _lib.load()
    act = P3M(**VALID)
    s = _lib.SystemDesc()
    for d in range(3):
        s.box[d] = 10.0
        s.periodic[d] = 1
    s.periodic[2] = 0
    s.skin = 0.4
    assert lib.p3mx_set_system(act._handle, ctypes.byref(s)) == 0
    pos = np.zeros((2, 3))
    q = np.array([1.0, -1.0])
    rc = lib.p3mx_activate(act._handle, 2, _lib.dptr(pos), _lib.dptr(q), 0)
    assert rc == 2
    assert b"CoulombP3M: requires periodicity (True, True, True)" in lib.p3mx_last_error(act._handle)
    f = np.zeros((2, 3))
    rc = lib.p3mx_long_range(act._handle, 2, _lib.dptr(pos), _lib.dptr(q), _lib.dptr(f),
                             None, None, _lib.P3MX_FORCES, None)
    assert rc == 2 and b"not activated" in lib.p3mx_last_error(act._handle)
    with pytest.raises(ValueError, match="box_l must be > 0"):
        s.box[0] = -1.0
        _lib.check(lib.p3mx_set_system(act._handle, ctypes.byref(s)), act._handle)


def test_neutrality_check_needs_no_gpu():
    lib = _lib.load()
    act = P3M(prefactor=1., accuracy=1e-3, mesh=8, cao=3, r_cut=1.0, alpha=1.0, tune=False)
    s = _lib.SystemDesc()
    for d in range(3):
        s.box[d] = 10.0
        s.periodic[d] = 1
    s.skin = 0.4
    lib.p3mx_set_system(act._handle, ctypes.byref(s))
    pos = np.zeros((2, 3))
    q = np.array([1.0, 1.0])
    rc = lib.p3mx_activate(act._handle, 2, _lib.dptr(pos), _lib.dptr(q), 0)
    assert rc == 2
    assert b"The system is not charge neutral" in lib.p3mx_last_error(act._handle)
