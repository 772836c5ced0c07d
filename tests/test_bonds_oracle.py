"""Bond restatement of the oracle (FENE, harmonic) pinned against the
reference test's own closed forms (testsuite/python/interactions_bonded.py:
harmonic_potential/force, fene_potential/force) and against -dE/dr."""
import numpy as np
import pytest

from oracle import oracle as O


def fene_potential(r, k, d_r_max, r_0):
    return -0.5 * k * d_r_max ** 2 * np.log(1 - ((r - r_0) / d_r_max) ** 2)


def fene_force(r, k, d_r_max, r_0):
    return k * (r - r_0) * d_r_max ** 2 / ((r - r_0) ** 2 - d_r_max ** 2)


def harmonic_potential(r, k, r_0):
    return 0.5 * k * (r - r_0) ** 2


def harmonic_force(r, k, r_0):
    return -k * (r - r_0)


@pytest.mark.parametrize("kind", ["fene", "harmonic"])
def test_dimer_scan_matches_reference_closed_forms(kind):
    """The reference test's dimer: p2 = p1 + axis * r over r in [0.01, cut)."""
    rng = np.random.default_rng(42)
    box = np.array([10.0] * 3)
    start = rng.random(3) * box
    axis = rng.random(3)
    axis /= np.linalg.norm(axis)
    if kind == "fene":
        k, d_r_max, r_0 = 23.15, 3.355, 1.1
        types = [(O.BOND_FENE, k, r_0, d_r_max)]
        cut = r_0 + d_r_max
        ef, ff = (lambda r: fene_potential(r, k, d_r_max, r_0),
                  lambda r: fene_force(r, k, d_r_max, r_0))
    else:
        k, r_0, r_cut = 5.0, 1.5, 3.355
        types = [(O.BOND_HARMONIC, k, r_0, r_cut)]
        cut = r_cut
        ef, ff = (lambda r: harmonic_potential(r, k, r_0), lambda r: harmonic_force(r, k, r_0))
    for r in np.linspace(0.01, cut, 11)[:-1]:
        pos = np.array([start, start + axis * r])
        f, e, v = O.bonds(box, pos, types, [(0, 0, 1)])
        np.testing.assert_allclose(e, ef(r), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(f[1], axis * ff(r), rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(f[0], -f[1], rtol=0, atol=0)
        # virial: F on p1 (x) (x1 - x2) = F_p2 (x) (x2 - x1)
        np.testing.assert_allclose(v, np.outer(f[1], axis * r), rtol=1e-12, atol=1e-13)
        # force = -dE/dr by central differences
        h = 1e-6
        num = -(ef(r + h) - ef(r - h)) / (2 * h)
        np.testing.assert_allclose(np.dot(f[1], axis), num, rtol=1e-6, atol=1e-6)
    with pytest.raises(RuntimeError, match="bond broken"):
        O.bonds(box, np.array([start, start + axis * cut * 1.01]), types, [(0, 0, 1)])
    with pytest.raises(RuntimeError):
        O.bonds(box, np.array([start, start]), types, [(0, 0, 1)])


def test_bond_across_the_periodic_boundary():
    box = np.array([8.0, 9.0, 10.0])
    pos = np.array([[0.2, 4.0, 9.9], [7.9, 4.5, 0.3]])
    types = [(O.BOND_HARMONIC, 3.0, 0.5, 0.0)]
    f, e, _ = O.bonds(box, pos, types, [(0, 0, 1)])
    d = np.array([0.3, -0.5, -0.4])  # minimum image x0 - x1
    r = np.linalg.norm(d)
    np.testing.assert_allclose(f[0], -3.0 * (r - 0.5) * d / r, rtol=1e-12)
    np.testing.assert_allclose(e, 1.5 * (r - 0.5) ** 2, rtol=1e-12)
