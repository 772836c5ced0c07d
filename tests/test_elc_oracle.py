"""The ELC restatement of the oracle, pinned on the reference's own golden
data (CPU only).

* testsuite/python/coulomb_mixed_periodicity.py:84-121: 285 charges in a
  10 x 10 x 12 box with a 3-unit gap; P3M (accuracy 1e-6, mesh 42 x 42 x 50,
  r_cut 3) + ELC (maxPWerror 1e-6) must give the MMM2D forces to 1e-5 and
  the MMM2D energy 216.640984711 to 1e-4.
* testsuite/python/p3m_madelung.py:236-277: the ionic sheet with ELC
  (maxPWerror 1e-6, gap 16) gives the Madelung constant of the square
  lattice to 1e-7 (energy per ion, metallic P3M with the test's parameters).
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _alpha_for(acc, r_cut, n, q2, box):
    """alpha with the real-space error acc / sqrt(2) (the tuner's split)."""
    lo, hi = 1e-3, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if O.rs_error(1.0, r_cut / box[0], n, q2, mid * box[0], box) > acc / np.sqrt(2.0):
            lo = mid
        else:
            hi = mid
    return hi


def test_elc_far_cut_and_modes():
    fc = O.elc_far_cut([10.0, 10.0, 12.0], 9.0, 1e-6)
    assert fc == pytest.approx(0.8)
    modes = O.elc_modes([10.0, 10.0, 12.0], fc)
    kinds = [m[0] for m in modes]
    # the cutoff is accumulated in steps of 1/L: 0.7999..., so frequency 9
    # ((9 - 1) / 10 = 0.8) is just outside, as in the reference
    assert fc < 0.8
    assert kinds.count(0) == 8 and kinds.count(1) == 8
    # p-major pq modes inside the quarter disc ((p-1)^2 + (q-1)^2) / 100 < fc^2
    assert kinds.count(2) == sum(1 for p in range(1, 10) for q in range(1, 10)
                                 if (0.1 * (p - 1)) ** 2 + (0.1 * (q - 1)) ** 2 < fc * fc)
    assert [m[1:3] for m in modes[16:19]] == [(1, 1), (1, 2), (1, 3)]
    with pytest.raises(RuntimeError, match="maxPWerror too small"):
        O.elc_far_cut([10.0, 10.0, 12.0], 11.99, 1e-300)


def test_elc_oracle_vs_mmm2d_golden():
    g = np.load(os.path.join(GOLD, "coulomb_mixed_periodicity.npz"))
    box, pos, q = g["box"], g["pos"], g["q"]
    assert pos[:, 2].min() >= 0.0 and pos[:, 2].max() <= box[2] - float(g["gap_size"])
    r_cut, acc = float(g["r_cut"]), float(g["accuracy"])
    alpha = _alpha_for(acc, r_cut, len(q), float(np.sum(q * q)), box)
    p = O.make_params(box, g["mesh"], 7, alpha, r_cut, 1.0)
    fk, ek, _ = O.p3m_kspace(p, pos, q)
    fr, er, _, _ = O.short_range(p, pos, q)
    fc = O.elc_far_cut(box, box[2] - float(g["gap_size"]), float(g["max_pw_error"]))
    fe, ee = O.elc(box, float(g["gap_size"]), pos, q, 1.0, fc)
    f = fk + fr + fe
    np.testing.assert_allclose(f, g["forces"], atol=float(g["force_atol"]), rtol=0)
    assert abs(ek + er[0] + ee - float(g["energy"])) < float(g["energy_atol"])
    # without the correction the slab forces are visibly wrong
    assert np.abs(fk + fr - g["forces"]).max() > 100 * float(g["force_atol"])


def test_elc_oracle_ionic_sheet_madelung():
    k = json.load(open(os.path.join(GOLD, "known_answers.json")))["madelung_sheet"]
    n = 2 * k["n_pairs"]
    box = np.array([n, n, 2.0 * n], dtype=float)
    jj, kk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    pos = np.stack([jj.ravel(), kk.ravel(), np.zeros(n * n)], axis=1).astype(float)
    q = (-1.0) ** (jj.ravel() + kk.ravel())
    p = O.make_params(box, k["mesh"], k["cao"], k["alpha"], k["r_cut"], 1.0)
    _, ek, _ = O.p3m_kspace(p, pos, q)
    _, er, _, _ = O.short_range(p, pos, q)
    gap = k["elc"]["gap_size"]
    fc = O.elc_far_cut(box, box[2] - gap, k["elc"]["maxPWerror"])
    _, ee = O.elc(box, gap, pos, q, 1.0, fc)
    e_ion = 2.0 * (ek + er[0] + ee) / len(q)
    np.testing.assert_allclose(e_ion, k["madelung"], rtol=k["energy_rtol"], atol=0)


def test_elc_oracle_gap_error():
    box = [10.0, 10.0, 13.0]
    pos = np.array([[1.0, 1.0, 1.0], [2.0, 2.0, 11.5]])
    with pytest.raises(RuntimeError, match="entered ELC gap region"):
        O.elc(box, 3.0, pos, [1.0, -1.0], 1.0, 0.5)
    # an uncharged particle may sit in the gap
    O.elc(box, 3.0, pos, [0.0, 0.0], 1.0, 0.5)


# --- dielectric contrasts and constant potential (oracle only; the CUDA path
# rejects contrasts) ---------------------------------------------------------

def test_elc_oracle_finite_potential_drop():
    """testsuite/python/elc.py:43-90: two charges between metallic walls
    (delta -1 / -1) with an applied potential difference of -3 and a
    vanishing Coulomb prefactor: energy -E (z1 q1 + z2 q2), force q E, with
    E = pot_diff / (L_z - gap)."""
    box = [10.0, 10.0, 13.0]
    pos = np.array([[0.0, 0.0, 1.0], [0.0, 0.0, 9.0]])
    q = np.array([1.0, -1.0])
    f, e = O.elc_system(box, 3.0, pos, q, 1e-100, 2.0, 2.0, 32, 5, 1e-3, delta_top=-1.0,
                        delta_bot=-1.0, const_pot=True, pot_diff=-3.0)
    e_field = -3.0 / 10.0
    assert e == pytest.approx(-e_field * (1.0 * 1.0 + 9.0 * -1.0), abs=1e-7)
    np.testing.assert_allclose(f[:, 2] / q, e_field, atol=1e-7)


def test_elc_oracle_metallic_walls_madelung():
    """testsuite/python/elc.py:107-145: a 12^3 rock-salt slab between
    metallic walls (delta -1 / -1, const_pot, no potential difference) is an
    infinite crystal: 2 E / N equals the cube Madelung constant to 1e-6."""
    n = 12
    idx = np.array(np.meshgrid(np.arange(n), np.arange(n), np.arange(n),
                               indexing="ij")).reshape(3, -1).T
    pos = idx + 0.5
    q = (-1.0) ** idx.sum(axis=1)
    gap = 0.4 * n
    _, e = O.elc_system([n, n, n + gap], gap, pos, q, 1.0, 1.18, 3.314, [60, 60, 84], 7, 3e-7,
                        delta_top=-1.0, delta_bot=-1.0, const_pot=True, pot_diff=0.0)
    np.testing.assert_allclose(2.0 * e / len(q), -1.74756459463318219, rtol=1e-6, atol=0)


def test_elc_oracle_dielectric_interface_vs_analytic():
    """testsuite/python/elc_vs_analytic.py:28-98: a +-q dipole along z at
    heights z in a 200 x 200 x 275 box (gap 75) above a dielectric interface
    (delta_mid_bot = 39/41): the z force on the lower charge and the energy
    equal the image-charge solution to 1e-4.  P3M: mesh 58 x 58 x 70, cao 4
    as the test; r_cut 60 and alpha from the real-space error of accuracy
    1e-7 (the test tunes them)."""
    box = np.array([200.0, 200.0, 275.0])
    pref, gap, dist, dmb, acc, r_cut = 2.0, 75.0, 1.0, 39.0 / 41.0, 1e-7, 60.0
    zs = np.linspace(0.1, 200.0 - 0.1 - dist, 12)
    qs = np.arange(-5.0, 5.1, 2.5)
    lo, hi = 1e-4, 5.0
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if O.rs_error(pref, r_cut / box[0], 2, 50.0, mid * box[0], box) > acc / np.sqrt(2.0):
            lo = mid
        else:
            hi = mid
    forces = np.empty((len(qs), len(zs)))
    energies = np.empty_like(forces)
    for a, qq in enumerate(qs):
        for b, z in enumerate(zs):
            pos = np.array([[100.0, 100.0, z], [100.0, 100.0, z + dist]])
            f, e = O.elc_system(box, gap, pos, [qq, -qq], pref, hi, r_cut, [58, 58, 70], 4, acc,
                                delta_bot=dmb)
            forces[a, b] = f[0, 2]
            energies[a, b] = e
    cq = pref * np.square(qs.reshape(-1, 1))
    f_ref = cq * (1 / dist ** 2 + dmb * (1 / np.square(2 * zs) - 1 / np.square(2 * zs + dist)))
    e_ref = cq * (-1 / dist + dmb * (1 / (4 * zs) - 1 / (2 * zs + dist) + 1 / (4 * (zs + dist))))
    np.testing.assert_allclose(energies, e_ref, atol=1e-4)
    np.testing.assert_allclose(forces, f_ref, atol=1e-4, rtol=1e-7)


def test_elc_oracle_system_without_contrast_is_p3m_plus_correction():
    g = np.load(os.path.join(GOLD, "coulomb_mixed_periodicity.npz"))
    box, pos, q = g["box"], g["pos"], g["q"]
    p = O.make_params(box, g["mesh"], 5, 2.0, 3.0, 1.0)
    fk, ek, _ = O.p3m_kspace(p, pos, q)
    fr, er, _, _ = O.short_range(p, pos, q)
    fc = O.elc_far_cut(box, box[2] - 3.0, 1e-5)
    fe, ee = O.elc(box, 3.0, pos, q, 1.0, fc)
    f, e = O.elc_system(box, 3.0, pos, q, 1.0, 2.0, 3.0, g["mesh"], 5, 1e-5)
    np.testing.assert_allclose(f, fk + fr + fe, rtol=0, atol=1e-12)
    assert e == pytest.approx(ek + er[0] + ee, rel=1e-14)
    with pytest.raises(RuntimeError, match="real-space cutoff too large"):
        O.elc_space_layer(3.0, 9.0, 3.0)
