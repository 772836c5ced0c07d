"""CPU tests: the FP64 oracle against the reference's golden vectors.

Mirrors the reference tests coulomb_cloud_wall.py, electrostatic_interactions.py,
p3m_madelung.py and lj.py (testsuite/python/), and pins the oracle's math
restatements against the reference's own headers (values in ref_math.npz).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden_systems import jittered_lattice, known, load, madelung_system


def test_math_against_reference_headers():
    g = load("ref_math.npz")
    xs = g["bspline_x"]
    for order in range(1, 8):
        for i in range(order):
            mine = [O.lib.oracle_bspline(order, i, float(x)) for x in xs]
            np.testing.assert_allclose(mine, g["bspline"][order, i], atol=1e-15, rtol=0)
    mine = [O.lib.oracle_as_erfc_part(float(d)) for d in g["as_erfc_d"]]
    np.testing.assert_allclose(mine, g["as_erfc"], rtol=1e-15, atol=0)
    mine = [O.lib.oracle_sinc(float(x)) for x in g["sinc_x"]]
    np.testing.assert_allclose(mine, g["sinc"], rtol=1e-15, atol=0)
    for cao in range(1, 8):
        for mi, m in enumerate(g["cot_meshes"]):
            for n in range(-m // 2, m // 2):
                v = O.lib.oracle_cotangent_sum(cao, n, 1.0 / m)
                assert abs(v - g["cot"][cao, mi, n + 32]) <= 1e-15 * abs(v)


def test_cloud_wall():
    g = load("coulomb_cloud_wall.npz")
    for pref in (3.0, 2.2):
        p = O.make_params(g["box"], g["mesh"], int(g["cao"]), float(g["alpha"]),
                          float(g["r_cut"]), pref)
        fk, ek, _ = O.p3m_kspace(p, g["pos"], g["q"])
        fr, er, _, _ = O.short_range(p, g["pos"], g["q"])
        np.testing.assert_allclose((fk + fr) / pref, g["forces"], atol=float(g["force_atol"]))
        assert abs((ek + er[0]) / pref - float(g["energy"])) < float(g["energy_atol"])


def test_two_charges_and_dipole_correction():
    ka = known()["two_charges"]
    pos, q, pref = np.array(ka["pos"]), np.array(ka["q"]), ka["prefactor"]
    p = O.make_params(ka["box"], ka["mesh"], ka["cao"], ka["alpha"], ka["r_cut"], pref)
    fk, ek, _ = O.p3m_kspace(p, pos, q)
    fr, er, _, _ = O.short_range(p, pos, q)
    e_met, f_met = ek + er[0], fk + fr
    assert abs(e_met - ka["energy_per_prefactor"] * pref) < ka["tol"]
    np.testing.assert_allclose(f_met[0], [ka["force_x_per_prefactor"] * pref, 0, 0], atol=ka["tol"])
    np.testing.assert_allclose(f_met[1], [-ka["force_x_per_prefactor"] * pref, 0, 0], atol=ka["tol"])
    V = ka["box"] ** 3
    dip = q @ pos
    for eps in 10.0 ** np.arange(-4, 5):
        p = O.make_params(ka["box"], ka["mesh"], ka["cao"], ka["alpha"], ka["r_cut"], pref,
                          epsilon=eps)
        fk, ek, _ = O.p3m_kspace(p, pos, q)
        corr = 4 * np.pi / V / (1 + 2 * eps)
        assert abs(ek + er[0] - (e_met + pref * corr * dip @ dip)) < ka["dipole_tol"]
        np.testing.assert_allclose(fk + fr, f_met - pref * np.outer(q, corr * dip),
                                   atol=ka["dipole_tol"])


@pytest.mark.parametrize("kind", ["wire", "sheet", "cube"])
def test_madelung(kind):
    box, pos, q, ka = madelung_system(kind)
    p = O.make_params(box, ka["mesh"], ka["cao"], ka["alpha"], ka["r_cut"], 1.0)
    fk, ek, vk = O.p3m_kspace(p, pos, q)
    fr, er, vc, _ = O.short_range(p, pos, q)
    n = len(q)
    e = 2 * (ek + er[0]) / n
    base = np.array(ka["base"], float)
    ref_p = ka["madelung"] * np.diag(base) / base.sum()
    assert abs(e - ka["madelung"]) <= ka["energy_rtol"] * abs(ka["madelung"])
    np.testing.assert_allclose(2 * (vk + vc) / n, ref_p, atol=5e-9, rtol=ka["pressure_rtol"])


def test_lj_system():
    g = load("lj_system.npz")
    p = O.make_params(float(g["box"]), 8, 7, 1.0, 1.0, 0.0)
    tab = O.pair_table(1, {(0, 0): dict(lj_eps=1.0, lj_sig=1.0, lj_cut=float(g["cut"]),
                                        lj_shift=float(g["shift"]))})
    f, _, _, _ = O.short_range(p, g["pos"], np.zeros(len(g["pos"])), None, 1, tab)
    diff = np.linalg.norm(f - g["forces"], axis=1)
    assert diff.mean() < 1e-7
    assert np.abs(f - g["forces"]).max() < 1e-5


def test_p3m_against_ewald():
    """Independent check: P3M (FP64 restatement) vs the direct Ewald sum."""
    box = 12.0
    pos, q = jittered_lattice(6, box, 0.3, seed=3)
    p = O.make_params(box, 48, 7, 1.2, 4.0, 1.0)
    fk, ek, _ = O.p3m_kspace(p, pos, q)
    fr, er, _, _ = O.short_range(p, pos, q)
    fe, ee = O.ewald([box] * 3, pos, q, 1.0, 0.6, 5.9, 16)
    rms = np.sqrt(((fk + fr - fe) ** 2).sum(1).mean())
    assert rms < 1e-5
    assert abs(ek + er[0] - ee) < 1e-5 * abs(ee)


def test_cell_grid_and_index():
    # C2 geometry: range 3.5 + 0.4 in a box of 128 gives 32^3 cells
    cg, cs = O.cell_grid(np.array([128.] * 3), 3.9)
    assert list(cg) == [32, 32, 32]
    cg, cs = O.cell_grid(np.array([20.] * 3), 3.0 + 0.4)
    assert list(cg) == [5, 5, 5]
    rng = np.random.default_rng(0)
    pos = rng.uniform(0, 20, (1000, 3))
    idx = O.cell_index(np.array([20.] * 3), 3.4, pos)
    cpos = np.floor(pos / 4.0).astype(int) + 1
    assert np.array_equal(idx, cpos[:, 0] + 7 * (cpos[:, 1] + 7 * cpos[:, 2]))


def test_error_estimates_match_known_tuning():
    """The two-charge parameters were tuned by the reference to 1e-7: the
    restated error estimate must confirm that accuracy for alpha given."""
    ka = known()["two_charges"]
    box = np.array([ka["box"]] * 3)
    L = box[0]
    rs = O.rs_error(1.0, ka["r_cut"] / L, 2, 2.0, ka["alpha"] * L, box)
    ks = O.ks_error(1.0, [ka["mesh"]] * 3, ka["cao"], 2, 2.0, ka["alpha"] * L, box)
    assert np.hypot(rs, ks) < 1.5 * ka["accuracy"]


def test_oracle_headline_parameters_rms_error_vs_ewald():
    """The FP64 restatement at the headline P3M parameters (mesh spacing 0.5,
    cao 7, r_cut 3.5, alpha 0.87024) on a box-24 system of the headline
    construction: rms Coulomb force error against the direct Ewald sum below
    the 1e-4 accuracy target (measured 5.9e-5; the error estimate says 7.9e-5)."""
    import bench
    pos, q, box = bench.make_workload(seed=3, box=24.0)
    fe, _ = O.ewald([box] * 3, pos, q, 1.0, 0.35, 9.9, 16)
    p = O.make_params([box] * 3, [48] * 3, 7, 0.8702383472846797, 3.5, 1.0)
    fk, _, _ = O.p3m_kspace(p, pos, q)
    fr, _, _, _ = O.short_range(p, pos, q)
    rms = np.sqrt((((fk + fr) - fe) ** 2).sum(1).mean())
    assert 2e-5 < rms < 1e-4
