"""GPU tests of the electrostatic layer correction (ELC) through the C ABI.

* the reference's testsuite/python/coulomb_mixed_periodicity.py:84-121: 285
  charges in a 10 x 10 x 12 box with a 3-unit gap; P3M (accuracy 1e-6, mesh
  42 x 42 x 50, r_cut 3, alpha and cao tuned) + ELC (maxPWerror 1e-6) against
  the MMM2D forces (1e-5) and energy (1e-4); resizing the box and back
  leaves forces and energy unchanged (1e-9);
* testsuite/python/p3m_madelung.py:236-277: ionic sheet with ELC, energy
  per ion equal to the square-lattice Madelung constant (rtol 1e-7);
* the ELC part alone (ELC run minus the bare P3M run) against the oracle's
  FP64 restatement, neutral and non-neutral, neutralize on and off
  (1e-9 of the largest force; energy 1e-9 relative);
* the gap check of testsuite/python/elc.py:92-104 (a charge in the gap,
  above and below, raises "entered ELC gap region").
"""
import ctypes
import json
import os

import numpy as np
import pytest

import espresso_b200 as eb
from espresso_b200 import _lib
from espresso_b200.electrostatics import ELC, P3M, P3MGPU
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _system(box, pos, q):
    s = eb.System(box_l=list(box))
    s.time_step = 0.01
    s.cell_system.skin = 0.0
    s.part.add(pos=pos, q=q)
    return s


@pytest.mark.parametrize("cls,ftol", [(P3M, None), (P3MGPU, 5e-5)])
def test_elc_vs_mmm2d_golden(cls, ftol):
    g = np.load(os.path.join(GOLD, "coulomb_mixed_periodicity.npz"))
    s = _system(g["box"], g["pos"], g["q"])
    p3m = cls(prefactor=1.0, accuracy=float(g["accuracy"]), mesh=[int(m) for m in g["mesh"]],
              r_cut=float(g["r_cut"]))
    elc = ELC(actor=p3m, maxPWerror=float(g["max_pw_error"]), gap_size=float(g["gap_size"]))
    s.electrostatics.solver = elc
    s.integrator.run(0)
    f1 = np.copy(s.part.all().f)
    e1 = s.analysis.energy()["total"]
    np.testing.assert_allclose(f1, g["forces"], atol=ftol or float(g["force_atol"]), rtol=0)
    assert abs(e1 - float(g["energy"])) < float(g["energy_atol"])
    # re-initialisation through a box change and back (coulomb_mixed_periodicity.py:67-82)
    box0 = np.copy(s.box_l)
    pos0 = np.copy(s.part.all().pos)
    for d in range(3):
        b = np.copy(box0)
        b[d] *= 1.05
        s.box_l = b
        s.part.all().pos = pos0 * (b / box0)
        s.integrator.run(0)
    s.box_l = box0
    s.part.all().pos = pos0
    s.integrator.run(0)
    np.testing.assert_allclose(s.part.all().f, f1, rtol=1e-9, atol=1e-12)
    assert abs(s.analysis.energy()["total"] - e1) <= 1e-9 * abs(e1)


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_elc_ionic_sheet_madelung(cls):
    k = json.load(open(os.path.join(GOLD, "known_answers.json")))["madelung_sheet"]
    n = 2 * k["n_pairs"]
    jj, kk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    pos = np.stack([jj.ravel(), kk.ravel(), np.zeros(n * n)], axis=1).astype(float)
    q = (-1.0) ** (jj.ravel() + kk.ravel())
    s = _system([n, n, 2.0 * n], pos, q)
    p3m = cls(prefactor=1.0, accuracy=k["accuracy"], mesh=k["mesh"], r_cut=k["r_cut"],
              cao=k["cao"], alpha=k["alpha"], tune=False)
    s.electrostatics.solver = ELC(actor=p3m, **k["elc"])
    e_ion = 2.0 * s.analysis.energy()["coulomb"] / len(q)
    np.testing.assert_allclose(e_ion, k["madelung"], rtol=k["energy_rtol"], atol=0)


@pytest.mark.parametrize("cls,neutral,neutralize", [(P3M, True, True), (P3M, False, True),
                                                     (P3M, False, False), (P3MGPU, True, True)])
def test_elc_part_vs_oracle(cls, neutral, neutralize):
    rng = np.random.default_rng(7)
    box = np.array([9.0, 11.0, 14.0])
    gap = 3.5
    n = 400
    pos = rng.uniform([0, 0, 0.2], [box[0], box[1], box[2] - gap - 0.2], (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    if not neutral:
        q[:3] = 2.0
    s = _system(box, pos, q)
    p3m = cls(prefactor=1.7, accuracy=1e-4, mesh=32, cao=5, r_cut=2.5, alpha=1.3, tune=False,
              check_neutrality=False)
    s.electrostatics.solver = p3m
    s.integrator.run(0)
    f0 = np.copy(s.part.all().f)
    e0 = s.analysis.energy()["coulomb"]
    elc = ELC(actor=p3m, maxPWerror=1e-7, gap_size=gap, neutralize=neutralize)
    s.electrostatics.solver = elc
    s.integrator.run(0)
    f1 = np.copy(s.part.all().f)
    e1 = s.analysis.energy()["coulomb"]
    fc = elc.far_cut
    assert fc == pytest.approx(O.elc_far_cut(box, box[2] - gap, 1e-7), rel=1e-12)
    nm = ctypes.c_int()
    assert _lib.load().p3mx_get_elc(elc._handle, None, None, ctypes.byref(nm)) == 0
    assert nm.value == len(O.elc_modes(box, fc)) > 20
    fo, eo = O.elc(box, gap, pos, q, 1.7, fc, neutralize=neutralize)
    np.testing.assert_allclose(f1 - f0, fo, atol=1e-9 * np.abs(fo).max(), rtol=0)
    assert abs((e1 - e0) - eo) <= 1e-9 * max(abs(eo), 1.0)
    # the bare actor again: no correction left on it
    s.electrostatics.solver = p3m
    s.integrator.run(0)
    np.testing.assert_allclose(s.part.all().f, f0, rtol=0, atol=1e-12)


def test_elc_gap_error():
    box = np.array([10.0, 10.0, 13.0])
    gap = 3.0
    s = _system(box, [[1.0, 1.0, 1.0], [5.0, 5.0, 9.0]], [1.0, -1.0])
    p3m = P3M(prefactor=1.0, accuracy=1e-3, mesh=32, cao=5, r_cut=2.0, alpha=1.5, tune=False)
    s.electrostatics.solver = ELC(actor=p3m, maxPWerror=1e-3, gap_size=gap)
    s.integrator.run(0)
    p1 = s.part.by_id(0)
    # positive direction (elc.py:92-97)
    p1.pos = [box[0] / 2, box[1] / 2, box[2] - gap / 2]
    with pytest.raises(Exception):
        s.analysis.energy()
    with pytest.raises(Exception, match="entered ELC gap region"):
        s.integrator.run(2)
    # negative direction (folded into the gap from below; elc.py:98-104)
    p1.pos = [box[0] / 2, box[1] / 2, -gap / 2]
    with pytest.raises(Exception, match="entered ELC gap region"):
        s.integrator.run(0)
    # back in the slab: usable again
    p1.pos = [1.0, 1.0, 1.0]
    s.integrator.run(0)


def test_elc_through_the_c_abi_long_range():
    """p3mx_long_range with ELC attached: forces and energy are the bare
    P3M ones plus the oracle's ELC part, the k-space virial is zero (the
    reference computes no ELC pressure), and p3mx_set_elc(NULL) detaches."""
    lib = _lib.load()
    rng = np.random.default_rng(11)
    box = np.array([10.0, 10.0, 15.0])
    gap = 4.0
    n = 300
    pos = rng.uniform([0, 0, 0.1], [box[0], box[1], box[2] - gap - 0.1], (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    p3m = P3M(prefactor=1.3, accuracy=1e-4, mesh=32, cao=5, r_cut=2.5, alpha=1.3, tune=False)
    p3m._set_system(box, 0.3, (True, True, True))
    p3m._activate(pos, q)
    h = p3m._handle
    flags = _lib.P3MX_FORCES | _lib.P3MX_ENERGY | _lib.P3MX_VIRIAL | _lib.P3MX_OVERWRITE

    def long_range():
        f = np.zeros((n, 3))
        e = np.zeros(1)
        v = np.zeros(9)
        _lib.check(lib.p3mx_long_range(h, n, _lib.dptr(pos), _lib.dptr(q), _lib.dptr(f),
                                       e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       flags, None), h)
        return f, e[0], v

    f0, e0, v0 = long_range()
    assert np.abs(v0).max() > 0.0
    c = _lib.ElcParams(maxPWerror=1e-6, gap_size=gap, far_cut=-1.0, neutralize=1)
    _lib.check(lib.p3mx_set_elc(h, ctypes.byref(c)), h)
    f1, e1, v1 = long_range()
    fc = ctypes.c_double()
    bh = ctypes.c_double()
    _lib.check(lib.p3mx_get_elc(h, ctypes.byref(fc), ctypes.byref(bh), None), h)
    assert bh.value == box[2] - gap
    fo, eo = O.elc(box, gap, pos, q, 1.3, fc.value)
    np.testing.assert_allclose(f1 - f0, fo, atol=1e-9 * np.abs(fo).max(), rtol=0)
    assert abs((e1 - e0) - eo) <= 1e-9 * max(abs(eo), 1.0)
    assert np.all(v1 == 0.0)
    _lib.check(lib.p3mx_set_elc(h, None), h)
    f2, e2, v2 = long_range()
    np.testing.assert_array_equal(f2, f0)
    assert e2 == e0
    assert lib.p3mx_get_elc(h, None, None, None) != 0


# --- dielectric contrasts and constant potential ------------------------------

def test_elc_finite_potential_drop():
    """testsuite/python/elc.py:43-104 (metallic walls, applied potential)."""
    gap = 3.0
    box = np.array([10.0, 10.0, 10.0 + gap])
    s = _system(box, [[0.0, 0.0, 1.0], [0.0, 0.0, 9.0]], [1.0, -1.0])
    p3m = P3M(prefactor=1e-100, mesh=32, cao=5, accuracy=1e-3)
    s.electrostatics.solver = ELC(actor=p3m, gap_size=gap, maxPWerror=1e-3, delta_mid_top=-1,
                                  delta_mid_bot=-1, const_pot=True, pot_diff=-3.0)
    u = s.analysis.energy()["coulomb"]
    e_field = -3.0 / (box[2] - gap)
    p1, p2 = s.part.by_id(0), s.part.by_id(1)
    assert u == pytest.approx(-e_field * (1.0 * 1.0 + 9.0 * -1.0), abs=1e-7)
    s.integrator.run(0)
    assert p1.f[2] / 1.0 == pytest.approx(e_field, abs=1e-7)
    assert p2.f[2] / -1.0 == pytest.approx(e_field, abs=1e-7)
    p1.pos = [box[0] / 2, box[1] / 2, box[2] - gap / 2]
    with pytest.raises(Exception, match="entered ELC gap region"):
        s.integrator.run(2)


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_elc_metallic_walls_madelung(cls):
    """testsuite/python/elc.py:107-145: rock salt between metallic walls."""
    n = 12
    idx = np.array(np.meshgrid(np.arange(n), np.arange(n), np.arange(n),
                               indexing="ij")).reshape(3, -1).T
    gap = 0.4 * n
    s = _system([n, n, n + gap], idx + 0.5, (-1.0) ** idx.sum(axis=1))
    p3m = cls(prefactor=1, mesh=[60, 60, 84], cao=7, r_cut=3.314, alpha=1.18, accuracy=3e-7,
              tune=False)
    s.electrostatics.solver = ELC(actor=p3m, gap_size=gap, maxPWerror=3e-7, delta_mid_top=-1,
                                  delta_mid_bot=-1, const_pot=True, pot_diff=0)
    u = 2.0 * s.analysis.energy()["coulomb"] / n ** 3
    np.testing.assert_allclose(u, -1.74756459463318219, rtol=1e-6, atol=0)


def test_elc_dielectric_interface_vs_analytic():
    """testsuite/python/elc_vs_analytic.py:28-98 (delta_mid_bot = 39/41);
    P3M mesh and cao of the test, r_cut 60 and the alpha of the real-space
    error 1e-7 (the test tunes them)."""
    box = np.array([200.0, 200.0, 275.0])
    gap, dist, dmb = 75.0, 1.0, 39.0 / 41.0
    zs = np.linspace(0.1, 200.0 - 0.1 - dist, 12)
    qs = np.arange(-5.0, 5.1, 2.5)
    s = _system(box, [[100.0, 100.0, 100.0], [100.0, 100.0, 100.0 + dist]], [qs[0], -qs[0]])
    s.cell_system.skin = 0.4
    p3m = P3M(prefactor=2.0, accuracy=1e-7, mesh=[58, 58, 70], cao=4, r_cut=60.0,
              alpha=0.05593284122999153, tune=False)
    s.electrostatics.solver = ELC(actor=p3m, gap_size=gap, maxPWerror=1e-7, delta_mid_bot=dmb,
                                  delta_mid_top=0.0)
    forces = np.empty((len(qs), len(zs)))
    energies = np.empty_like(forces)
    p1, p2 = s.part.by_id(0), s.part.by_id(1)
    for a, qq in enumerate(qs):
        p1.q, p2.q = qq, -qq
        for b, z in enumerate(zs):
            p1.pos = [100.0, 100.0, z]
            p2.pos = [100.0, 100.0, z + dist]
            s.integrator.run(0)
            forces[a, b] = p1.f[2]
            energies[a, b] = s.analysis.energy()["total"]
    cq = 2.0 * np.square(qs.reshape(-1, 1))
    f_ref = cq * (1 / dist ** 2 + dmb * (1 / np.square(2 * zs) - 1 / np.square(2 * zs + dist)))
    e_ref = cq * (-1 / dist + dmb * (1 / (4 * zs) - 1 / (2 * zs + dist) + 1 / (4 * (zs + dist))))
    np.testing.assert_allclose(energies, e_ref, atol=1e-4)
    np.testing.assert_allclose(forces, f_ref, atol=1e-4, rtol=1e-7)


def test_elc_contrast_vs_oracle():
    """A neutral slab between two dielectric walls (delta 0.5 below, -0.3
    above): forces and energy against the oracle's elc_system."""
    rng = np.random.default_rng(5)
    box = np.array([9.0, 10.0, 14.0])
    gap = 3.5
    n = 240
    pos = rng.uniform([0, 0, 0.05], [box[0], box[1], box[2] - gap - 0.05], (n, 3))
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    s = _system(box, pos, q)
    p3m = P3M(prefactor=1.3, accuracy=1e-4, mesh=32, cao=5, r_cut=2.0, alpha=1.6, tune=False)
    s.electrostatics.solver = ELC(actor=p3m, gap_size=gap, maxPWerror=1e-6, delta_mid_bot=0.5,
                                  delta_mid_top=-0.3)
    s.integrator.run(0)
    f = s.part.all().f
    e = s.analysis.energy()["coulomb"]
    fo, eo = O.elc_system(box, gap, pos, q, 1.3, 1.6, 2.0, 32, 5, 1e-6, delta_bot=0.5,
                          delta_top=-0.3)
    np.testing.assert_allclose(f, fo, atol=1e-9 * np.abs(fo).max(), rtol=0)
    assert e == pytest.approx(eo, rel=1e-8, abs=1e-8)
    # a net charge with a non-metallic contrast is rejected
    s.part.by_id(0).q = 2.0
    with pytest.raises(Exception, match="non-neutral"):
        s.integrator.run(0)
