"""Parameter handling of the DipolarP3M actor mirror (no GPU needed: the
handle only validates and stores until it is activated).  Messages and
exception types follow src/python/espressomd/magnetostatics.py:44-160 and
the C++ checks of p3m/common.hpp:95-150 and dp3m.impl.hpp:85-92."""
import pickle

import pytest

from espresso_b200.magnetostatics import DipolarP3M

BASE = dict(prefactor=1.0, accuracy=1e-4, mesh=16, cao=5, r_cut=2.0, alpha=1.0, tune=False)


def _with(**kw):
    p = dict(BASE)
    p.update(kw)
    return p


@pytest.mark.parametrize("kw, exc, msg", [
    (dict(prefactor=-1.0), ValueError, "Parameter 'prefactor' must be > 0"),
    (dict(prefactor="a"), ValueError, "Parameter 'prefactor' should be a float"),
    (dict(accuracy=-1.0), ValueError, "Parameter 'accuracy' must be > 0"),
    (dict(r_cut=-2.0), ValueError, "Parameter 'r_cut' must be > 0"),
    (dict(alpha=-2.0), ValueError, "Parameter 'alpha' must be > 0"),
    (dict(cao=0), ValueError, "Parameter 'cao' must be >= 1 and <= 7"),
    (dict(cao=8), ValueError, "Parameter 'cao' must be >= 1 and <= 7"),
    (dict(cao=7, mesh=4), ValueError, "Parameter 'cao' cannot be larger than 'mesh'"),
    (dict(mesh=[16, 16, 8]), ValueError, "DipolarP3M requires a cubic mesh"),
    (dict(mesh=[16, 16]), ValueError, "integer or integer list of length 3"),
    (dict(mesh_off=[-0.5, 0.5, 0.5]), ValueError, "Parameter 'mesh_off' must be >= 0 and <= 1"),
    (dict(mesh_off=[0.5, 0.5]), ValueError, "has to be a \\(3,\\) array_like"),
    (dict(epsilon=-1.0), ValueError, "Parameter 'epsilon' must be >= 0"),
    (dict(epsilon="x"), ValueError, "has to be a float or 'metallic'"),
    (dict(timings=0), ValueError, "Parameter 'timings' must be > 0"),
    (dict(timings=1.5), TypeError, "Parameter 'timings' has to be an integer"),
    (dict(tune=1), TypeError, "Parameter 'tune' has to be a boolean"),
    (dict(unknown=1), RuntimeError, "Parameter 'unknown' is not a valid parameter"),
])
def test_invalid_parameters(kw, exc, msg):
    with pytest.raises(exc, match=msg):
        DipolarP3M(**_with(**kw))


def test_accuracy_is_required():
    with pytest.raises(RuntimeError, match="Parameter 'accuracy' is missing"):
        DipolarP3M(prefactor=1.0)


def test_defaults_and_view_before_activation():
    act = DipolarP3M(prefactor=2.0, accuracy=1e-3)
    p = act.get_params()
    assert p["mesh"] == [-1, -1, -1] and p["cao"] == -1 and not p["is_tuned"]
    assert p["epsilon"] == 0.0 and p["mesh_off"] == [0.5, 0.5, 0.5]
    assert p["single_precision"] is False and p["timings"] == 10 and p["tune"] is True
    fixed = DipolarP3M(**_with(epsilon="metallic", mesh=[16, 16, 16]))
    q = fixed.get_params()
    assert q["is_tuned"] and q["mesh"] == [16, 16, 16] and q["cao"] == 5
    assert q["epsilon"] == 0.0 and fixed.get_magnetostatics_prefactor() == 1.0


def test_pickle_round_trip_keeps_parameters():
    act = DipolarP3M(**_with(epsilon=1.5, mesh_off=[0.25, 0.5, 0.75]))
    back = pickle.loads(pickle.dumps(act))
    assert back.get_params()["mesh_off"] == [0.25, 0.5, 0.75]
    assert back.epsilon == 1.5 and back.cao == 5 and back.r_cut == 2.0
