"""GPU tests of the pair bonds (FENE, harmonic) through the C ABI.

The dimer scans follow the reference test testsuite/python/interactions_bonded.py
(same bond parameters, distances, force / energy / pressure checks, breakage
and same-position errors); the chain melt compares the full force path (FENE
+ WCA + P3M) with the FP64 oracle, for the plain FP64 path (1e-9 relative)
and the FP32-mixed path (2e-5 relative, the P3M tolerance of the other
parity tests; the bond forces themselves are FP64 in both).
"""
import numpy as np
import pytest

import espresso_b200 as eb
from espresso_b200.electrostatics import P3M, P3MGPU
from espresso_b200.interactions import FeneBond, HarmonicBond
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _fene(r, k, d_r_max, r_0):
    return (k * (r - r_0) * d_r_max ** 2 / ((r - r_0) ** 2 - d_r_max ** 2),
            -0.5 * k * d_r_max ** 2 * np.log(1 - ((r - r_0) / d_r_max) ** 2))


def _harmonic(r, k, r_0):
    return -k * (r - r_0), 0.5 * k * (r - r_0) ** 2


@pytest.mark.parametrize("kind", ["fene", "harmonic"])
def test_dimer_scan_as_the_reference_test(kind):
    rng = np.random.default_rng(42)
    box_l = 10.0
    start = rng.random(3) * box_l
    axis = rng.random(3)
    axis /= np.linalg.norm(axis)
    s = eb.System(box_l=[box_l] * 3)
    s.time_step = 0.2
    s.cell_system.skin = 0.4
    p1 = s.part.add(pos=start, type=0)
    p2 = s.part.add(pos=start, type=0)
    if kind == "fene":
        k, d_r_max, r_0 = 23.15, 3.355, 1.1
        bond = FeneBond(k=k, d_r_max=d_r_max, r_0=r_0)
        cut = r_0 + d_r_max
        ref = lambda r: _fene(r, k, d_r_max, r_0)  # noqa: E731
    else:
        k, r_0, r_cut = 5.0, 1.5, 3.355
        bond = HarmonicBond(k=k, r_0=r_0, r_cut=r_cut)
        cut = r_cut
        ref = lambda r: _harmonic(r, k, r_0)  # noqa: E731
    s.bonded_inter.add(bond)
    p1.bonds = ((bond, p2),)
    for dist in np.linspace(0.01, cut, 11)[:-1]:
        p2.pos = p1.pos + axis * dist
        s.integrator.run(recalc_forces=True, steps=0)
        f_ref, e_ref = ref(dist)
        e_sim = s.analysis.energy()["total"]
        f0, f1 = np.copy(p1.f), np.copy(p2.f)
        assert abs(e_sim - e_ref) < 1e-7
        np.testing.assert_allclose(f0, -f1, rtol=1e-12)
        np.testing.assert_almost_equal(f1, axis * f_ref)
        p_expected = np.dot(f1, axis * dist) / 3.0 / s.volume()
        assert abs(s.analysis.pressure()["total"] - p_expected) < 1e-12
        np.testing.assert_allclose(s.analysis.pressure_tensor()["total"],
                                   np.outer(f1, axis * dist) / s.volume(), atol=1e-12)
    p2.pos = p1.pos + axis * cut * 1.01
    with pytest.raises(Exception, match="bond broken"):
        s.integrator.run(recalc_forces=True, steps=0)
    p2.pos = p1.pos
    with pytest.raises(Exception):
        s.integrator.run(recalc_forces=True, steps=0)


def _chain_melt(n_chains=9, length=12, box=12.0, seed=3):
    """Charged FENE chains along x (bond length 0.97) on a y-z lattice with
    jitter, charges alternating +1/-1 along each chain (neutral)."""
    rng = np.random.default_rng(seed)
    pos, q, bonds = [], [], []
    side = int(np.ceil(np.sqrt(n_chains)))
    for c in range(n_chains):
        y0, z0 = (c % side + 0.5) * box / side, (c // side + 0.5) * box / side
        x0 = rng.uniform(0, box)
        for b in range(length):
            pos.append([x0 + 0.97 * b, y0, z0] + rng.uniform(-0.05, 0.05, 3))
            q.append(1.0 if b % 2 == 0 else -1.0)
            if b > 0:
                i = c * length + b
                bonds.append((0, i - 1, i))
    return np.array(pos), np.array(q), np.array(bonds, dtype=np.int32)


@pytest.mark.parametrize("cls,rtol", [(P3M, 1e-9), (P3MGPU, 2e-5)])
def test_charged_chain_melt_vs_oracle(cls, rtol):
    box = 12.0
    pos, q, bonds = _chain_melt(box=box)
    k, d_r_max = 30.0, 1.5
    s = eb.System(box_l=[box] * 3)
    s.time_step = 0.005
    s.cell_system.skin = 0.3
    s.part.add(pos=pos, q=q)
    s.non_bonded_inter[0, 0].wca.set_params(epsilon=1.0, sigma=1.0)
    fene = FeneBond(k=k, d_r_max=d_r_max)
    s.bonded_inter.add(fene)
    for _, i, j in bonds:
        s.part.by_id(i).add_bond((fene, j))
    s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-3, mesh=24, cao=5, alpha=1.0,
                                  r_cut=3.0, tune=False)
    tab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
    p = O.make_params([box] * 3, [24] * 3, 5, 1.0, 3.0, 1.0)
    cur = pos
    for step in range(3):
        if step:
            s.integrator.run(5)
            cur = s.part.all().pos
        else:
            s.integrator.run(0, recalc_forces=True)
        f = s.part.all().f
        fk, ek, _ = O.p3m_kspace(p, cur, q)
        fr, er, _, _ = O.short_range(p, cur, q, tab=tab)
        fb, eb_, vb = O.bonds([box] * 3, cur, [(O.BOND_FENE, k, 0.0, d_r_max)], bonds)
        fo = fk + fr + fb
        np.testing.assert_allclose(f, fo, atol=rtol * np.abs(fo).max(), rtol=0)
        en = s.analysis.energy()
        assert abs(en["bonded"] - eb_) <= 1e-10 * abs(eb_)
        np.testing.assert_allclose(s.analysis.pressure_tensor()["bonded"] * box ** 3, vb,
                                   rtol=1e-10, atol=1e-10)


def test_bonds_only_system_and_changes():
    """Bonds without any pair interaction run on the short-range handle;
    replacing a particle's bonds and clearing them take effect."""
    s = eb.System(box_l=[10.0] * 3)
    s.time_step = 0.01
    s.part.add(pos=[[1.0, 1.0, 1.0], [2.2, 1.0, 1.0], [2.2, 2.3, 1.0]])
    h = HarmonicBond(k=4.0, r_0=1.0)
    s.bonded_inter.add(h)
    s.part.by_id(0).add_bond((h, 1))
    s.integrator.run(0, recalc_forces=True)
    np.testing.assert_allclose(s.part.by_id(0).f, [0.8, 0.0, 0.0], rtol=1e-12)
    np.testing.assert_allclose(s.part.by_id(2).f, 0.0, atol=0)
    s.part.by_id(0).bonds = ((h, 2),)
    s.integrator.run(0, recalc_forces=True)
    fb, _, _ = O.bonds([10.0] * 3, s.part.all().pos, [(O.BOND_HARMONIC, 4.0, 1.0, 0.0)],
                       [(0, 0, 2)])
    np.testing.assert_allclose(s.part.all().f, fb, rtol=1e-12, atol=1e-14)
    s.bonded_inter.clear()
    s.integrator.run(0, recalc_forces=True)
    np.testing.assert_allclose(s.part.all().f, 0.0, atol=0)
