"""GPU parity tests of the P3M + short-range path through the C ABI.

Structure follows the reference tests (testsuite/python/coulomb_cloud_wall.py,
electrostatic_interactions.py, p3m_madelung.py, coulomb_tuning.py, lj.py):
the same systems and tolerances against the golden fixtures, plus tighter
element-wise comparisons with the FP64 oracle.  Tolerances: the plain FP64
GPU path must agree with the oracle to 1e-9 (relative to the force scale);
the FP32-mixed path to 2e-5 relative (FP32 mesh/FFT arithmetic).
"""
import ctypes

import numpy as np
import pytest

import espresso_b200 as eb
from espresso_b200 import _lib
from espresso_b200.electrostatics import P3M, P3MGPU
from oracle import oracle as O
from tests.golden_systems import jittered_lattice, known, load, madelung_system

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-9
FP32_RTOL = 2e-5


def make_system(box, pos, q, skin=0.4):
    s = eb.System(box_l=box)
    s.time_step = 0.01
    s.cell_system.skin = skin
    s.part.add(pos=pos, q=q)
    return s


def oracle_total(box, pos, q, mesh, cao, alpha, r_cut, pref, epsilon=0.0):
    p = O.make_params(box, mesh, cao, alpha, r_cut, pref, epsilon=epsilon)
    fk, ek, vk = O.p3m_kspace(p, pos, q)
    fr, er, vc, _ = O.short_range(p, pos, q)
    return fk + fr, ek + er[0], vk + vc


@pytest.mark.parametrize("cls,rtol", [(P3M, FP64_RTOL), (P3MGPU, FP32_RTOL)])
def test_cloud_wall(cls, rtol):
    g = load("coulomb_cloud_wall.npz")
    pref = 3.0 if cls is P3M else 2.2
    s = make_system(g["box"], g["pos"], g["q"])
    s.electrostatics.solver = cls(prefactor=pref, accuracy=float(g["accuracy"]),
                                  mesh=[int(m) for m in g["mesh"]], cao=int(g["cao"]),
                                  alpha=float(g["alpha"]), r_cut=float(g["r_cut"]), tune=False)
    s.integrator.run(0)
    f = s.part.all().f
    e = s.analysis.energy()["total"]
    # reference test tolerances against the stored data
    np.testing.assert_allclose(f / pref, g["forces"], atol=float(g["force_atol"]))
    assert abs(e / pref - float(g["energy"])) < float(g["energy_atol"])
    # element-wise against the oracle
    fo, eo, _ = oracle_total(g["box"], g["pos"], g["q"], g["mesh"], int(g["cao"]),
                             float(g["alpha"]), float(g["r_cut"]), pref)
    scale = np.abs(fo).max()
    np.testing.assert_allclose(f, fo, atol=rtol * scale, rtol=0)
    assert abs(e - eo) <= rtol * abs(eo) + 1e-12


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_two_charges_metallic_and_dipole(cls):
    ka = known()["two_charges"]
    pref = ka["prefactor"]
    pos, q = np.array(ka["pos"]), np.array(ka["q"])
    s = make_system(ka["box"], pos, q)
    kw = dict(prefactor=pref, accuracy=ka["accuracy"], mesh=[ka["mesh"]] * 3, cao=ka["cao"],
              r_cut=ka["r_cut"], alpha=ka["alpha"], tune=False)
    s.electrostatics.solver = cls(epsilon="metallic", **kw)
    s.integrator.run(0)
    e_met = s.analysis.energy()["coulomb"]
    f_met = s.part.all().f
    assert abs(e_met - ka["energy_per_prefactor"] * pref) < ka["tol"]
    np.testing.assert_allclose(f_met[0], [ka["force_x_per_prefactor"] * pref, 0, 0], atol=ka["tol"])
    np.testing.assert_allclose(f_met[1], [-ka["force_x_per_prefactor"] * pref, 0, 0], atol=ka["tol"])
    if cls is P3MGPU:
        return
    V = ka["box"] ** 3
    dip = q @ pos
    for eps in 10.0 ** np.arange(-4, 5):
        s.electrostatics.clear()
        s.electrostatics.solver = cls(epsilon=float(eps), **kw)
        s.integrator.run(0)
        corr = 4 * np.pi / V / (1 + 2 * eps)
        e = s.analysis.energy()["coulomb"]
        np.testing.assert_allclose(e, e_met + pref * corr * dip @ dip, atol=ka["dipole_tol"])
        np.testing.assert_allclose(s.part.all().f, f_met - pref * np.outer(q, corr * dip),
                                   atol=ka["dipole_tol"])


@pytest.mark.parametrize("kind", ["wire", "sheet", "cube"])
@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_madelung(kind, cls):
    box, pos, q, ka = madelung_system(kind)
    params = dict(mesh=ka["mesh"], cao=ka["cao"], r_cut=ka["r_cut"], alpha=ka["alpha"],
                  accuracy=ka["accuracy"])
    if kind == "cube" and cls is P3MGPU:
        params = dict(ka["gpu_params"])
    s = make_system(box, pos, q)
    s.electrostatics.solver = cls(prefactor=1.0, tune=False, **params)
    n = len(q)
    V = float(np.prod(box))
    energy = 2.0 * s.analysis.energy()["coulomb"] / n
    p_tensor = 2.0 * s.analysis.pressure_tensor()["coulomb"] * V / n
    p_scalar = 2.0 * s.analysis.pressure()["coulomb"] * V / n
    base = np.array(ka["base"], float)
    ref_p = ka["madelung"] * np.diag(base) / base.sum()
    np.testing.assert_allclose(energy, ka["madelung"], atol=0, rtol=ka["energy_rtol"])
    np.testing.assert_allclose(p_scalar, np.trace(ref_p) / 3.0, atol=1e-12, rtol=ka["pressure_rtol"])
    np.testing.assert_allclose(p_tensor, ref_p, atol=5e-9, rtol=ka["pressure_rtol"])


def _handle_compute(cls, box, pos, q, mesh, cao, alpha, r_cut, pref=1.0):
    act = cls(prefactor=pref, accuracy=1e-4, mesh=mesh, cao=cao, alpha=alpha, r_cut=r_cut,
              tune=False, check_neutrality=False)
    act._set_system(np.broadcast_to(box, (3,)), 0.4, (True, True, True))
    act._activate(pos, q)
    lib = _lib.load()
    f = np.zeros((len(q), 3))
    e = np.zeros(1)
    v = np.zeros(9)
    rc = lib.p3mx_long_range(act._handle, len(q), _lib.dptr(_lib.as_f64(pos)),
                             _lib.dptr(_lib.as_f64(q)), _lib.dptr(f),
                             e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             _lib.P3MX_FORCES | _lib.P3MX_ENERGY | _lib.P3MX_VIRIAL |
                             _lib.P3MX_OVERWRITE, None)
    _lib.check(rc, act._handle)
    mesh_out = np.zeros(int(np.prod(np.broadcast_to(mesh, (3,)))))
    _lib.check(lib.p3mx_copy_mesh(act._handle, mesh_out.ctypes.data_as(
        ctypes.POINTER(ctypes.c_double)), mesh_out.size), act._handle)
    return act, f, e[0], v.reshape(3, 3), mesh_out


@pytest.mark.parametrize("mesh_off", [0.25, 0.5, 0.75, (0.1, 0.6, 0.9)])
@pytest.mark.parametrize("cls,rtol", [(P3M, FP64_RTOL), (P3MGPU, FP32_RTOL)])
def test_mesh_off_vs_oracle(mesh_off, cls, rtol):
    """Non-default mesh offsets (P3MParameters::mesh_off, p3m/common.hpp:
    156-171: grid position pos * ai - mesh_off, CA-mesh origin ld_pos):
    charge mesh and k-space forces, energy and virial equal the oracle's."""
    box = np.array([11.0, 10.0, 12.0])
    rng = np.random.default_rng(17)
    n = 300
    pos = rng.uniform(0.0, 1.0, (n, 3)) * box
    q = rng.choice([-1.0, 1.0], n)
    q -= q.mean()
    mesh = [22, 20, 24]
    off = np.broadcast_to(np.asarray(mesh_off, dtype=float), (3,))
    act = cls(prefactor=1.3, accuracy=1e-4, mesh=mesh, cao=5, alpha=1.2, r_cut=2.5,
              mesh_off=list(off), tune=False, check_neutrality=False)
    act._set_system(box, 0.4, (True, True, True))
    act._activate(pos, q)
    lib = _lib.load()
    f = np.zeros((n, 3))
    e = np.zeros(1)
    v = np.zeros(9)
    rc = lib.p3mx_long_range(act._handle, n, _lib.dptr(_lib.as_f64(pos)), _lib.dptr(_lib.as_f64(q)),
                             _lib.dptr(f), e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             _lib.P3MX_FORCES | _lib.P3MX_ENERGY | _lib.P3MX_VIRIAL |
                             _lib.P3MX_OVERWRITE, None)
    _lib.check(rc, act._handle)
    mesh_gpu = np.zeros(int(np.prod(mesh)))
    _lib.check(lib.p3mx_copy_mesh(act._handle, mesh_gpu.ctypes.data_as(
        ctypes.POINTER(ctypes.c_double)), mesh_gpu.size), act._handle)
    p = O.make_params(box, mesh, 5, 1.2, 2.5, 1.3, mesh_off=off)
    fo, eo, vo, rho = O.p3m_kspace(p, pos, q, want_mesh=True)
    np.testing.assert_allclose(mesh_gpu, rho.ravel(), atol=rtol * np.abs(rho).max() * 10, rtol=0)
    np.testing.assert_allclose(f, fo, atol=rtol * np.abs(fo).max(), rtol=0)
    assert abs(e[0] - eo) <= rtol * abs(eo) * 10 + 1e-12
    np.testing.assert_allclose(v.reshape(3, 3), vo, atol=rtol * np.abs(vo).max() * 10, rtol=0)


@pytest.mark.parametrize("eps", [0.5, 1.0, 80.0])
def test_fp32_mixed_dipole_correction_vs_oracle(eps):
    """The FP32-mixed actor with a finite dielectric (epsilon != metallic:
    the dipole force and energy terms of p3m.cpp:481-488, 540-547, 575-577)
    against the FP64 oracle, element-wise at the FP32-mixed tolerance."""
    box = 14.0
    pos, q = jittered_lattice(8, box, 0.3, seed=31)  # 512 ions
    pos[:40, 2] += 2.0  # a net dipole moment
    s = make_system([box] * 3, pos, q)
    s.electrostatics.solver = P3MGPU(prefactor=1.0, accuracy=1e-4, mesh=32, cao=6, r_cut=3.0,
                                     alpha=1.1, epsilon=eps, tune=False)
    s.integrator.run(0)
    f = s.part.all().f
    e = s.analysis.energy()["coulomb"]
    fo, eo, _ = oracle_total([box] * 3, pos, q, 32, 6, 1.1, 3.0, 1.0, epsilon=eps)
    np.testing.assert_allclose(f, fo, atol=FP32_RTOL * np.abs(fo).max(), rtol=0)
    assert abs(e - eo) <= FP32_RTOL * abs(eo) + 1e-9


def test_mixed_observables_vs_oracle():
    """P3MX_MIXED_OBSERVABLES: energies and virials of the FP32-mixed actor
    from its own FP32 kernels (not the default FP64 observables engine)
    against the FP64 oracle, at the FP32-mixed tolerance (x 10 for sums)."""
    box = 13.0
    pos, q = jittered_lattice(8, box, 0.25, seed=41)
    act = P3MGPU(prefactor=1.7, accuracy=1e-4, mesh=32, cao=5, r_cut=3.0, alpha=1.2,
                 tune=False)
    s = make_system([box] * 3, pos, q)
    s.electrostatics.solver = act
    lib = _lib.load()
    n = len(q)
    f = np.zeros((n, 3))
    e3 = np.zeros(3)
    v27 = np.zeros(27)
    flags = (_lib.P3MX_FORCES | _lib.P3MX_ENERGY | _lib.P3MX_VIRIAL | _lib.P3MX_OVERWRITE |
             _lib.P3MX_MIXED_OBSERVABLES)
    rc = lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q), None, _lib.dptr(f),
                         e3.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                         v27.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), flags, None)
    _lib.check(rc, act._handle)
    p = O.make_params([box] * 3, 32, 5, 1.2, 3.0, 1.7)
    fk, ek, vk = O.p3m_kspace(p, pos, q)
    fr, er, vc, _ = O.short_range(p, pos, q)
    # energy3: real-space Coulomb, k-space, non-bonded; virial27: the same
    assert abs(e3[1] - ek) <= FP32_RTOL * 10 * abs(ek)
    assert abs(e3[0] - er[0]) <= FP32_RTOL * 10 * abs(er[0])
    np.testing.assert_allclose(v27[9:18].reshape(3, 3), vk, atol=FP32_RTOL * 10 * np.abs(vk).max(),
                               rtol=0)
    np.testing.assert_allclose(v27[0:9].reshape(3, 3), vc, atol=FP32_RTOL * 10 * np.abs(vc).max(),
                               rtol=0)
    np.testing.assert_allclose(f, fk + fr, atol=FP32_RTOL * np.abs(fk + fr).max(), rtol=0)


@pytest.mark.parametrize("cao", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("cls,rtol", [(P3M, FP64_RTOL), (P3MGPU, FP32_RTOL)])
def test_kspace_elementwise_vs_oracle(cao, cls, rtol):
    """Charge mesh, k-space forces, energy and virial vs the FP64 oracle on a
    ragged non-cubic mesh (16 x 22 x 18; 22 and 18 exercise radix 11 and 3)."""
    box = np.array([10.0, 12.0, 11.0])
    rng = np.random.default_rng(cao)
    n = 333
    pos = rng.uniform(-1.0, 1.0, (n, 3)) * box + box / 2  # some outside the box
    q = rng.choice([-1.0, 1.0, 2.0, -2.0, 0.0], n)
    q -= q.mean()
    mesh = [16, 22, 18]
    _, f, e, v, mesh_gpu = _handle_compute(cls, box, pos, q, mesh, cao, 1.1, 2.5)
    p = O.make_params(box, mesh, cao, 1.1, 2.5, 1.0)
    fo, eo, vo, rho = O.p3m_kspace(p, pos, q, want_mesh=True)
    np.testing.assert_allclose(mesh_gpu, rho.ravel(), atol=rtol * np.abs(rho).max() * 10, rtol=0)
    np.testing.assert_allclose(f, fo, atol=rtol * np.abs(fo).max(), rtol=0)
    assert abs(e - eo) <= rtol * abs(eo) * 10 + 1e-12
    np.testing.assert_allclose(v, vo, atol=rtol * np.abs(vo).max() * 10, rtol=0)


def test_assignment_is_deterministic():
    box = 20.0
    pos, q = jittered_lattice(12, box, 0.2, seed=7)
    act, f1, e1, _, m1 = _handle_compute(P3MGPU, box, pos, q, 32, 7, 1.0, 3.0)
    lib = _lib.load()
    for _ in range(2):
        f2 = np.zeros_like(f1)
        rc = lib.p3mx_long_range(act._handle, len(q), _lib.dptr(_lib.as_f64(pos)),
                                 _lib.dptr(_lib.as_f64(q)), _lib.dptr(f2), None, None,
                                 _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE, None)
        _lib.check(rc, act._handle)
        m2 = np.zeros_like(m1)
        lib.p3mx_copy_mesh(act._handle, m2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), m2.size)
        assert np.array_equal(m1, m2)
        assert np.array_equal(f1, f2)


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_resort_rebuilds_to_the_same_forces(cls):
    """cell_system.resort() (p3mx_resort) makes the next force calculation
    rebuild the cell and Verlet lists; on an unchanged configuration the
    rebuilt lists give bitwise the same forces."""
    box = 16.0
    pos, q = jittered_lattice(10, box, 0.2, seed=11)
    s = make_system([box] * 3, pos, q)
    s.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0, cutoff=2.5,
                                                      shift="auto")
    s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-4, mesh=32, cao=5, r_cut=3.0,
                                  alpha=1.0, tune=False)
    s.integrator.run(0)
    f1 = s.part.all().f.copy()
    s.cell_system.resort()
    s.integrator.run(0)
    assert np.array_equal(s.part.all().f, f1)


def test_fp32_real_space_pair_force_vs_fp64_formula():
    """The FP32 real-space Coulomb force of CoulombP3M::pair_force
    (p3m.hpp:146-163: exp(-(alpha r)^2) (AS(alpha r)/r + 2 alpha/sqrt(pi)) / r^2
    times q1 q2 d, with the A&S 7.1.26 exp(x^2) erfc(x) of AS_erfc_part.hpp)
    against the same formula in FP64, over r in (0.2, r_cut): isolated pairs,
    one per lattice site of a large box, through p3mx_short_range.  The FP32
    kernel forms exp(-(alpha r)^2) as 2^(-alpha^2 log2(e) r^2) with the
    hardware ex2 approximation and uses approximate reciprocals; its force
    stays within 4e-6 of the FP64 value relative to the force at that r, and
    the forces on the two particles of a pair cancel to round-off."""
    alpha, r_cut = 0.87, 3.5
    n_side, spacing = 10, 8.0  # pairs farther apart than r_cut + skin
    box = n_side * spacing
    rng = np.random.default_rng(5)
    n_pairs = n_side ** 3
    r = np.linspace(0.2, r_cut - 0.01, n_pairs)
    u = rng.normal(size=(n_pairs, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    site = (np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
            + 0.5) * spacing
    pos = np.empty((2 * n_pairs, 3))
    pos[0::2] = site - 0.5 * r[:, None] * u
    pos[1::2] = site + 0.5 * r[:, None] * u
    qa = rng.choice([-2.0, -1.0, 1.0, 2.0], n_pairs)
    q = np.empty(2 * n_pairs)
    q[0::2] = qa
    q[1::2] = -qa
    act = P3MGPU(prefactor=1.0, accuracy=1e-4, mesh=32, cao=5, alpha=alpha, r_cut=r_cut,
                 tune=False)
    act._set_system(np.array([box] * 3), 0.4, (True, True, True))
    act._activate(pos, q)
    lib = _lib.load()
    f = np.zeros((2 * n_pairs, 3))
    rc = lib.p3mx_short_range(act._handle, len(q), _lib.dptr(pos), _lib.dptr(q), None,
                              _lib.dptr(f), None, None,
                              _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE, None)
    _lib.check(rc, act._handle)
    d = pos[0::2] - pos[1::2]
    ar = alpha * r
    t = 1.0 / (1.0 + 0.3275911 * ar)
    asp = t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 +
                                                                        t * 1.061405429))))
    fac = qa * (-qa) * np.exp(-ar ** 2) * (asp / r + 2 * alpha / np.sqrt(np.pi)) / r ** 2
    f_ref = fac[:, None] * d
    rel = np.linalg.norm(f[0::2] - f_ref, axis=1) / np.linalg.norm(f_ref, axis=1)
    assert rel.max() < 4e-6, rel.max()
    np.testing.assert_allclose(f[1::2], -f[0::2], rtol=0, atol=1e-12 * np.abs(f).max())


def test_lj_system():
    g = load("lj_system.npz")
    s = eb.System(box_l=[float(g["box"])] * 3)
    s.time_step = 0.1
    s.cell_system.skin = float(g["skin"])
    s.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0,
                                                      cutoff=float(g["cut"]), shift="auto")
    s.part.add(pos=g["pos"])
    for _ in range(2):  # build the Verlet list, then reuse it
        s.integrator.run(0, recalc_forces=True)
        f = s.part.all().f
        assert np.linalg.norm(f - g["forces"], axis=1).mean() < 1e-7
        assert np.abs(f - g["forces"]).max() < 1e-5


def test_cell_index_bit_exact_and_pair_set():
    """Cell assignment equals position_to_cell_index; the Verlet pair set
    equals the oracle's link-cell pair set (check_non_bonded_loop_trace)."""
    box = 20.0
    rng = np.random.default_rng(11)
    n = 3000
    pos = rng.uniform(0, box, (n, 3))
    pos[:5] = [[0.0, 0.0, 0.0], [box - 1e-12, 5.0, 5.0], [4.0, 4.0, 4.0], [8.0, 12.0, 16.0],
               [19.999999999, 0.0, 3.4]]
    q = rng.choice([-1.0, 1.0], n)
    s = make_system([box] * 3, pos, q)
    act = P3M(prefactor=1.0, accuracy=1e-3, mesh=16, cao=3, alpha=1.0, r_cut=3.0, tune=False,
              check_neutrality=False)
    s.electrostatics.solver = act
    lib = _lib.load()
    cell = np.zeros(n, dtype=np.int32)
    _lib.check(lib.p3mx_cell_index(act._handle, n, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   cell.ctypes.data_as(ctypes.POINTER(ctypes.c_int))), act._handle)
    cg = np.zeros(3, dtype=np.int32)
    cs = np.zeros(3)
    lib.p3mx_cell_grid(act._handle, cg.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                       cs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    cg_o, cs_o = O.cell_grid(np.array([box] * 3), 3.0 + 0.4)
    assert list(cg) == list(cg_o)
    np.testing.assert_array_equal(cell, O.cell_index(np.array([box] * 3), 3.4, pos))
    cap = 200 * n
    pairs = np.zeros(2 * cap, dtype=np.int32)
    cnt = ctypes.c_size_t()
    _lib.check(lib.p3mx_verlet_pairs(act._handle, n, pos.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None,
                                     pairs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cap,
                                     ctypes.byref(cnt)), act._handle)
    mine = {tuple(p) for p in pairs[:2 * cnt.value].reshape(-1, 2)}
    ref = {tuple(sorted(p)) for p in O.verlet_pairs([box] * 3, 0.4, 3.0, pos, q)}
    assert mine == ref


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_tuning(cls):
    """coulomb_tuning.py: tune to accuracy 5e-4, forces within 2e-3."""
    g = load("coulomb_tuning.npz")
    s = make_system(g["box"], g["pos"], g["q"])
    act = cls(prefactor=1.0, accuracy=float(g["accuracy"]), tune=True, verbose=False)
    s.electrostatics.solver = act
    assert act.is_tuned
    assert act.get_params()["accuracy"] <= float(g["accuracy"])
    s.integrator.run(0)
    np.testing.assert_allclose(s.part.all().f, g["forces"], atol=float(g["force_atol"]))


def test_error_estimate_matches_oracle():
    lib = _lib.load()
    box = np.array([20.0, 20.0, 20.0])
    for mesh, cao, aL, rcL in [(32, 5, 12.0, 0.15), (22, 7, 7.75, 0.445), (64, 3, 30.0, 0.05)]:
        m = np.array([mesh] * 3, dtype=np.int32)
        rs = ctypes.c_double()
        ks = ctypes.c_double()
        rc = lib.p3mx_error_estimate(m.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cao, 2000,
                                     2000.0, aL, rcL, box.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                     1.0, ctypes.byref(rs), ctypes.byref(ks))
        assert rc == 0
        # device exp/pow/cos differ from the host libm by ulps, amplified by
        # the cancellation inside the aliasing sum
        np.testing.assert_allclose(ks.value, O.ks_error(1.0, mesh, cao, 2000, 2000.0, aL, box),
                                   rtol=1e-7)
        np.testing.assert_allclose(rs.value, O.rs_error(1.0, rcL, 2000, 2000.0, aL, box), rtol=1e-14)


def test_fp32_accuracy_vs_ewald_c1_like():
    """2000 ions in L=20 with mesh 32 and cao 5, r_cut and alpha tuned to
    accuracy 1e-4 (at the fixed r_cut 3.0 the error estimate cannot go below
    1.1e-3): the FP32-mixed path's rms force error against the FP64 Ewald
    sum stays at the P3M error level, and within 5% of the FP64 oracle's."""
    box = 20.0
    pos, q = jittered_lattice(10, box, 0.2, seed=1)  # 1000 ions
    pos2, q2 = jittered_lattice(10, box, 0.2, seed=2)
    pos = np.vstack([pos, pos2 + 0.5 * box / 10])
    q = np.concatenate([q, -q2])
    s = make_system([box] * 3, pos, q)
    act = P3MGPU(prefactor=1.0, accuracy=1e-4, mesh=32, cao=5, tune=True, verbose=False)
    s.electrostatics.solver = act
    s.integrator.run(0)
    f = s.part.all().f
    fe, ee = O.ewald([box] * 3, pos, q, 1.0, 0.35, 9.9, 18)
    rms = np.sqrt(((f - fe) ** 2).sum(1).mean())
    est = act.get_params()["accuracy"]
    assert rms < 3 * max(est, 1e-4)
    fo, _, _ = oracle_total([box] * 3, pos, q, 32, 5, act.alpha, act.r_cut, 1.0)
    rms_o = np.sqrt(((fo - fe) ** 2).sum(1).mean())
    assert abs(rms - rms_o) < 0.05 * rms_o + 1e-6


def test_host_staging_chunks_accumulate_and_device_pointers():
    """Host-pointer calls stage through pinned memory in chunks (several
    chunks here): overwrite and accumulate modes and the device-pointer path
    give the same forces bit for bit."""
    import torch
    box = 64.0
    pos, q = jittered_lattice(48, box, 0.3, seed=11)  # 110592 ions
    shifts = np.repeat([[0., 0., 0.], [0.31, 0.17, 0.05], [0.6, 0.44, 0.29]], len(q), 0)
    pos = np.ascontiguousarray(np.tile(pos, (3, 1)) + shifts)
    q = np.ascontiguousarray(np.tile(q, 3))  # 331776 ions: 8 MB of positions
    act = P3MGPU(prefactor=1.0, accuracy=1e-3, mesh=64, cao=5, alpha=0.9, r_cut=2.0,
                 tune=False, check_neutrality=False)
    act._set_system(np.full(3, box), 0.4, (True, True, True))
    act._activate(pos, q)
    lib = _lib.load()
    n = len(q)
    f_ow = np.zeros((n, 3))
    flags = _lib.P3MX_FORCES | _lib.P3MX_OVERWRITE
    _lib.check(lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q), None,
                               _lib.dptr(f_ow), None, None, flags, None), act._handle)
    assert np.all(np.isfinite(f_ow)) and np.abs(f_ow).max() > 0
    f0 = np.random.default_rng(3).normal(size=(n, 3))
    f_acc = f0.copy()
    _lib.check(lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q), None,
                               _lib.dptr(f_acc), None, None, _lib.P3MX_FORCES, None), act._handle)
    assert np.array_equal(f_acc, f0 + f_ow)
    dp = torch.from_numpy(pos).cuda()
    dq = torch.from_numpy(q).cuda()
    df = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(lib.p3mx_forces(act._handle, n, dp.data_ptr(), dq.data_ptr(), None, df.data_ptr(),
                               None, None, flags | _lib.P3MX_DEVICE_PTRS, None), act._handle)
    torch.cuda.synchronize()
    assert np.array_equal(df.cpu().numpy(), f_ow)
    # unchanged charges are not staged again: a changed chunk must be sent
    # (one + and one - ion swap sign, in different 4 MB chunks)
    q2 = q.copy()
    i_plus = int(np.flatnonzero(q2 > 0)[1000])
    i_minus = int(np.flatnonzero(q2 < 0)[-1000])
    q2[i_plus], q2[i_minus] = -q2[i_plus], -q2[i_minus]
    # host call right after a host call: computed first with the staged
    # charges, found changed, computed again
    _lib.check(lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q), None,
                               _lib.dptr(f_acc), None, None, flags, None), act._handle)
    f2s = np.zeros((n, 3))
    _lib.check(lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q2), None,
                               _lib.dptr(f2s), None, None, flags, None), act._handle)
    f2 = np.zeros((n, 3))
    _lib.check(lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q2), None,
                               _lib.dptr(f2), None, None, flags, None), act._handle)
    assert np.array_equal(f2s, f2)
    dq2 = torch.from_numpy(q2).cuda()
    torch.cuda.synchronize()
    _lib.check(lib.p3mx_forces(act._handle, n, dp.data_ptr(), dq2.data_ptr(), None, df.data_ptr(),
                               None, None, flags | _lib.P3MX_DEVICE_PTRS, None), act._handle)
    torch.cuda.synchronize()
    assert not np.array_equal(f2, f_ow)
    assert np.array_equal(df.cpu().numpy(), f2)
    # and back to the original charges through the host path again
    f3 = np.zeros((n, 3))
    _lib.check(lib.p3mx_forces(act._handle, n, _lib.dptr(pos), _lib.dptr(q), None,
                               _lib.dptr(f3), None, None, flags, None), act._handle)
    assert np.array_equal(f3, f_ow)


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_headline_parameters_rms_error_vs_ewald(cls):
    """The P3M parameters of the 2^20-ion headline workload (mesh spacing 0.5,
    cao 7, r_cut 3.5, alpha 0.87024 from its tuning to accuracy 1e-4) on a
    box-24 system of the same construction and density (6912 ions, mesh 48):
    the rms Coulomb force error against the FP64 direct Ewald sum stays below
    the 1e-4 target that the headline metric is quoted at."""
    import bench
    pos, q, box = bench.make_workload(seed=3, box=24.0)
    s = make_system([box] * 3, pos, q)
    s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-4, mesh=48, cao=7, r_cut=3.5,
                                  alpha=0.8702383472846797, tune=False)
    s.integrator.run(0)
    f = s.part.all().f
    # Ewald: real space erfc(0.35 * 9.9) ~ 1e-6, k space exp(-k^2/4a^2) < 1e-15
    fe, _ = O.ewald([box] * 3, pos, q, 1.0, 0.35, 9.9, 16)
    rms = np.sqrt(((f - fe) ** 2).sum(1).mean())
    assert rms < 1e-4
    assert rms > 1e-6  # the comparison resolves the P3M discretisation error


@pytest.mark.parametrize("cls,rtol", [(P3M, FP64_RTOL), (P3MGPU, FP32_RTOL)])
def test_forces_after_moves_across_the_boundary(cls, rtol):
    """Forces after moves that keep the Verlet list (below skin/2) or force
    a rebuild, with ions crossing the periodic boundary and unfolded input
    coordinates, equal the oracle's on the moved configuration: the
    FP32-mixed kernel's cell-relative geometry must follow the particles."""
    box = 12.0
    pos, q = jittered_lattice(8, box, 0.2, seed=21)  # 512 ions
    pos[:8, 0] = box - 0.03
    pos[8:16, 1] = 0.02
    pos[16:24, 2] = box - 0.01
    s = make_system([box] * 3, pos, q)
    s.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0, cutoff=2.5,
                                                      shift="auto")
    s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-3, mesh=24, cao=5, alpha=1.0,
                                  r_cut=3.0, tune=False)
    s.integrator.run(0, recalc_forces=True)
    shift = -((1.0 / 2.5) ** 12 - (1.0 / 2.5) ** 6)
    tab = O.pair_table(1, {(0, 0): dict(lj_eps=1.0, lj_sig=1.0, lj_cut=2.5, lj_shift=shift)})
    p = O.make_params([box] * 3, [24] * 3, 5, 1.0, 3.0, 1.0)
    rng = np.random.default_rng(5)
    cur = pos.copy()
    for step in range(4):
        d = rng.uniform(-0.05, 0.05, cur.shape)
        d[:8, 0] = 0.06    # across x = box
        d[8:16, 1] = -0.05  # across y = 0
        d[16:24, 2] = 0.04  # across z = box
        cur = cur + d       # unfolded coordinates, outside [0, box) for some
        s.part.all().pos = cur
        s.integrator.run(0, recalc_forces=True)
        f = s.part.all().f
        fk, _, _ = O.p3m_kspace(p, cur, q)
        fr, _, _, _ = O.short_range(p, cur, q, None, 1, tab)
        ref = fk + fr
        np.testing.assert_allclose(f, ref, atol=rtol * np.abs(ref).max() * 10, rtol=0)


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_changed_types_and_charges_between_host_calls(cls):
    """Host-pointer force calls compute first with the charges and types
    staged by the previous call and compare them with the new arrays on the
    host meanwhile; changed types or charges must still give, bit for bit,
    the forces of a fresh system built with the new values."""
    box = 10.0
    pos, q = jittered_lattice(8, box, 0.2, seed=31)  # 512 ions
    rng = np.random.default_rng(8)
    t1 = rng.integers(0, 2, len(q)).astype(np.int32)
    t2 = t1.copy()
    t2[:40] = 1 - t2[:40]
    q2 = q.copy()
    q2[100:110] = -q2[100:110]

    def system(types, charges):
        s = make_system([box] * 3, pos, charges)
        s.part.all().type = types
        for (a, b), eps in {(0, 0): 1.0, (0, 1): 0.5, (1, 1): 2.0}.items():
            s.non_bonded_inter[a, b].lennard_jones.set_params(epsilon=eps, sigma=1.0,
                                                              cutoff=2.5, shift="auto")
        s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-3, mesh=20, cao=5, alpha=1.0,
                                      r_cut=3.0, tune=False)
        return s

    def forces(s):
        s.integrator.run(0, recalc_forces=True)
        return s.part.all().f.copy()

    s = system(t1, q)
    forces(s)
    forces(s)  # staged charges and types unchanged
    s.part.all().type = t2
    f_t = forces(s)
    assert np.array_equal(f_t, forces(system(t2, q)))
    s.part.all().q = q2
    f_q = forces(s)
    assert np.array_equal(f_q, forces(system(t2, q2)))
    assert not np.array_equal(f_t, f_q)


@pytest.mark.parametrize("cls", [P3M, P3MGPU])
def test_checkpoint_keeps_tuned_parameters(cls):
    """A pickled system (as the reference's checkpointing) restores the
    solver with its tuned parameters, without tuning again, and gives the
    same forces bit for bit."""
    import pickle
    from espresso_b200.interactions import FeneBond
    box = 12.0
    pos, q = jittered_lattice(8, box, 0.2, seed=41)
    s = make_system([box] * 3, pos, q)
    s.non_bonded_inter[0, 0].wca.set_params(epsilon=1.0, sigma=1.0)
    fene = FeneBond(k=10.0, d_r_max=2.0)
    s.bonded_inter.add(fene)
    s.part.by_id(0).add_bond((fene, 1))
    s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-3, tune=True, verbose=False,
                                  timings=2)
    s.integrator.run(0, recalc_forces=True)
    f0 = s.part.all().f
    s2 = pickle.loads(pickle.dumps(s))
    p1, p2 = s.electrostatics.solver.get_params(), s2.electrostatics.solver.get_params()
    for k in ("mesh", "cao", "r_cut", "alpha", "mesh_off", "prefactor", "accuracy"):
        assert p1[k] == p2[k], k
    assert p1["is_tuned"] and p2["is_tuned"] and p2["tune"] is False
    s2.integrator.run(0, recalc_forces=True)
    assert np.array_equal(s2.part.all().f, f0)
    assert len(s2.part.by_id(0).bonds) == 1


@pytest.mark.parametrize("mesh,cao", [([8, 10, 12], 7), ([6, 8, 10], 5), ([8, 8, 8], 8 - 1)])
@pytest.mark.parametrize("cls,rtol", [(P3M, FP64_RTOL), (P3MGPU, FP32_RTOL)])
def test_kspace_meshes_smaller_than_a_brick_tile(mesh, cao, cls, rtol):
    """Meshes smaller than one brick tile (brick + cao - 1 points): the
    assignment tiles overlap themselves (multi-pass flush by wrap class) and
    the ghost layers of the field mesh cover most of it; charge mesh, forces
    and energy still match the FP64 oracle."""
    box = np.array([7.0, 8.0, 9.0])
    rng = np.random.default_rng(cao + mesh[0])
    n = 150
    pos = rng.uniform(0.0, 1.0, (n, 3)) * box
    q = rng.choice([-1.0, 1.0], n)
    q -= q.mean()
    _, f, e, v, mesh_gpu = _handle_compute(cls, box, pos, q, mesh, cao, 0.9, 2.0)
    p = O.make_params(box, mesh, cao, 0.9, 2.0, 1.0)
    fo, eo, vo, rho = O.p3m_kspace(p, pos, q, want_mesh=True)
    np.testing.assert_allclose(mesh_gpu, rho.ravel(), atol=rtol * np.abs(rho).max() * 10, rtol=0)
    np.testing.assert_allclose(f, fo, atol=rtol * np.abs(fo).max() * 10, rtol=0)
    assert abs(e - eo) <= rtol * abs(eo) * 10 + 1e-12
    np.testing.assert_allclose(v, vo, atol=rtol * np.abs(vo).max() * 10, rtol=0)


def test_degenerate_inputs():
    """Edge cases of the reference's own checks and of empty work: tuning
    without charged particles raises its runtime error (p3m.cpp:769-771);
    an untuned actor on all-zero charges gives the LJ forces alone; a
    single ion (neutrality check off) gets a finite force; a system without
    particles runs."""
    box = 10.0
    pos, _ = jittered_lattice(6, box, 0.2, seed=51)  # 216 particles
    zero = np.zeros(len(pos))
    s = make_system([box] * 3, pos, zero)
    with pytest.raises(Exception, match="no charged particles"):
        s.electrostatics.solver = P3MGPU(prefactor=1.0, accuracy=1e-3, tune=True, verbose=False)
    s.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0, cutoff=2.5,
                                                      shift="auto")
    s.integrator.run(0, recalc_forces=True)
    f_lj = s.part.all().f
    # (the FP32-mixed actor evaluates LJ in FP32 too)
    for cls, tol in ((P3M, 1e-12), (P3MGPU, FP32_RTOL * np.abs(f_lj).max())):
        s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-3, mesh=16, cao=5, alpha=1.0,
                                      r_cut=2.5, tune=False, check_neutrality=False)
        s.integrator.run(0, recalc_forces=True)
        np.testing.assert_allclose(s.part.all().f, f_lj, rtol=0, atol=tol)
        s.electrostatics.clear()
    one = make_system([box] * 3, np.array([[1.0, 2.0, 3.0]]), np.array([1.0]))
    one.electrostatics.solver = P3MGPU(prefactor=1.0, accuracy=1e-3, mesh=16, cao=5, alpha=1.0,
                                       r_cut=2.5, tune=False, check_neutrality=False)
    one.integrator.run(0, recalc_forces=True)
    assert np.all(np.isfinite(one.part.all().f))
    assert np.abs(one.part.all().f).max() < 1e-3  # the self force of one ion vanishes
    empty = eb.System(box_l=[box] * 3)
    empty.time_step = 0.01
    empty.non_bonded_inter[0, 0].lennard_jones.set_params(epsilon=1.0, sigma=1.0, cutoff=2.5)
    empty.integrator.run(2)
    assert empty.analysis.energy()["total"] == 0.0
