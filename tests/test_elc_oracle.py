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
