"""ELC actor parameter checks (CPU; no device work): the messages of the
reference's elc_data constructor (core/electrostatics/elc.cpp:1056-1102) and
of the Python actor (src/python/espressomd/electrostatics.py:345-365)."""
import pytest

from espresso_b200.electrostatics import ELC, P3M


@pytest.fixture(scope="module")
def p3m():
    return P3M(prefactor=1.0, accuracy=1e-3, epsilon=1.0)


@pytest.mark.parametrize("kw,exc,msg", [
    (dict(far_cut=0.0), ValueError, "Parameter 'far_cut' must be > 0"),
    (dict(maxPWerror=0.0), ValueError, "Parameter 'maxPWerror' must be > 0"),
    (dict(gap_size=-1.0), ValueError, "Parameter 'gap_size' must be > 0"),
    (dict(pot_diff=3.0), ValueError, "Parameter 'const_pot' must be True when 'pot_diff'"),
    (dict(delta_mid_top=1.5), ValueError, "Parameter 'delta_mid_top' must be >= -1 and <= \\+1"),
    (dict(delta_mid_bot=-1.5), ValueError, "Parameter 'delta_mid_bot' must be >= -1 and <= \\+1"),
    (dict(delta_mid_bot=-1.0, delta_mid_top=-1.0), ValueError,
     "two parallel metallic boundaries requires the const_pot option"),
    (dict(far_cut="x"), TypeError, "far_cut has to be a float"),
    (dict(maxPWerror="x"), TypeError, "maxPWerror has to be a float"),
    (dict(neutralize=1), TypeError, "neutralize has to be a bool"),
])
def test_invalid_parameters(p3m, kw, exc, msg):
    params = dict(actor=p3m, gap_size=2.0, maxPWerror=1e-4)
    params.update(kw)
    with pytest.raises(exc, match=msg):
        ELC(**params)


def test_required_keys_and_defaults(p3m):
    with pytest.raises(ValueError, match="At least the following keys"):
        ELC(actor=p3m, gap_size=2.0)
    elc = ELC(actor=p3m, gap_size=2.0, maxPWerror=1e-4)
    assert elc.neutralize is True and elc.delta_mid_top == 0.0 and elc.const_pot is False
    assert elc.actor is p3m
    # adapt_epsilon_elc: the base P3M is metallic under ELC
    assert p3m.epsilon == 0.0
    # const_pot without a dielectric contrast has no effect (elc.cpp:1063)
    ELC(actor=p3m, gap_size=2.0, maxPWerror=1e-4, const_pot=True, pot_diff=1.0)


def test_pickle_round_trip(p3m):
    """A pickled ELC actor restores its parameters and its base actor
    (checkpointing as the reference's script interface does)."""
    import pickle
    elc = ELC(actor=p3m, gap_size=2.5, maxPWerror=1e-5, far_cut=0.3, neutralize=False)
    back = pickle.loads(pickle.dumps(elc))
    assert isinstance(back, ELC) and back is not elc
    for key in ("gap_size", "maxPWerror", "far_cut", "neutralize", "delta_mid_top"):
        assert back.get_params()[key] == elc.get_params()[key]
    assert type(back.actor) is type(p3m) and back.actor.prefactor == p3m.prefactor
