"""GPU tests of the dipolar P3M actor (DipolarP3M) against the oracle's
restatement of magnetostatics/dp3m.cpp and the reference's own data.

Tolerances: the FP64 path against the FP64 oracle differs only by rounding
(fixed-point mesh assignment with 2^-51 resolution, a different FFT and
summation order): 1e-9 relative to the largest component.  The FP32 path
(single_precision=True: FP32 mesh, FFT and real-space pair terms, FP64
sums) carries FP32 rounding: 1e-4 relative rms.  Reference data are checked with
the tolerances of the reference's tests (p3m_madelung.py,
dipolar_mdlc_p3m_scafacos_p2nfft.py).
"""
import itertools
import json
import os

import numpy as np
import pytest
from scipy.special import zeta

import espresso_b200 as eb
from espresso_b200.magnetostatics import DipolarP3M
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
MAG = json.load(open(os.path.join(GOLD, "known_answers.json")))["magnetic"]


def _system(L, pos, dip, skin=0.4):
    s = eb.System(box_l=[L] * 3)
    s.time_step = 0.01
    s.cell_system.skin = skin
    s.part.add(pos=pos, dip=dip)
    return s


def _random(n, L, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, L, (n, 3)), rng.normal(size=(n, 3))


def _forces_torques_energy(s):
    s.integrator.run(0)
    e = s.analysis.energy()["dipolar"]
    return s.part.all().f, s.part.all().torque_lab, e


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("accuracy", [1e-4, 1e-7])  # A&S erfc / exact erfc branch
def test_fp64_matches_oracle(accuracy):
    L, n = 10.0, 60
    pos, dip = _random(n, L, 3)
    args = dict(prefactor=1.3, alpha=0.9, r_cut=3.0, mesh=16, cao=5, accuracy=accuracy)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(tune=False, **args)
    f, t, e = _forces_torques_energy(s)
    fo, to, eo = O.dp3m(L, pos, dip, args["prefactor"], args["alpha"], args["r_cut"],
                        args["mesh"], args["cao"], accuracy)
    assert _rel(f, fo) < 1e-9
    assert _rel(t, to) < 1e-9
    assert e == pytest.approx(eo, rel=1e-10)


@pytest.mark.parametrize("cao", [1, 2, 3, 4, 6, 7])
def test_fp64_every_order_and_mesh_off(cao):
    L, n = 12.0, 40
    pos, dip = _random(n, L, 10 + cao)
    off = (0.25, 0.5, 0.75)
    args = dict(prefactor=1.0, alpha=0.8, r_cut=3.5, mesh=24, cao=cao, accuracy=1e-4)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(tune=False, mesh_off=list(off), **args)
    f, t, e = _forces_torques_energy(s)
    fo, to, eo = O.dp3m(L, pos, dip, 1.0, 0.8, 3.5, 24, cao, 1e-4, mesh_off=off)
    assert _rel(f, fo) < 1e-9
    assert _rel(t, to) < 1e-9
    assert e == pytest.approx(eo, rel=1e-10)


def test_non_magnetic_particles_and_surface_term():
    """Particles without a moment feel nothing and change nothing; a
    non-metallic boundary adds the surface term (calc_surface_term)."""
    L, n = 10.0, 50
    pos, dip = _random(n, L, 21)
    dip[::3] = 0.0
    args = dict(prefactor=1.0, alpha=0.9, r_cut=3.0, mesh=16, cao=6, accuracy=1e-4)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(tune=False, epsilon=2.0, **args)
    f, t, e = _forces_torques_energy(s)
    keep = np.any(dip != 0, axis=1)
    fo, to, eo = O.dp3m(L, pos[keep], dip[keep], 1.0, 0.9, 3.0, 16, 6, 1e-4, epsilon=2.0)
    assert np.all(f[~keep] == 0) and np.all(t[~keep] == 0)
    assert _rel(f[keep], fo) < 1e-9
    assert _rel(t[keep], to) < 1e-9
    assert e == pytest.approx(eo, rel=1e-10)


def test_fp32_mesh_path():
    L, n = 10.0, 60
    pos, dip = _random(n, L, 4)
    args = dict(prefactor=1.0, alpha=0.9, r_cut=3.0, mesh=32, cao=5, accuracy=1e-4)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(tune=False, single_precision=True, **args)
    f, t, e = _forces_torques_energy(s)
    fo, to, eo = O.dp3m(L, pos, dip, 1.0, 0.9, 3.0, 32, 5, 1e-4)

    def rms_rel(a, b):
        return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
    assert rms_rel(f, fo) < 1e-4
    assert rms_rel(t, to) < 1e-4
    assert e == pytest.approx(eo, rel=1e-5)


def test_fp32_path_cell_grid():
    """The FP32 path on a box of 4 cells per axis (the real-space pairs from
    the cell-relative offsets and the entries' cell-offset fields, no
    minimum-image arithmetic), against the oracle."""
    L, n = 16.0, 300
    pos, dip = _random(n, L, 11)
    args = dict(prefactor=1.0, alpha=0.9, r_cut=3.0, mesh=32, cao=5, accuracy=1e-4)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(tune=False, single_precision=True, **args)
    f, t, e = _forces_torques_energy(s)
    fo, to, eo = O.dp3m(L, pos, dip, 1.0, 0.9, 3.0, 32, 5, 1e-4)

    def rms_rel(a, b):
        return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
    assert rms_rel(f, fo) < 1e-4
    assert rms_rel(t, to) < 1e-4
    assert e == pytest.approx(eo, rel=1e-5)


def test_deterministic_and_repeatable():
    L, n = 10.0, 80
    pos, dip = _random(n, L, 5)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(prefactor=1.0, tune=False, alpha=0.9, r_cut=3.0, mesh=16,
                                         cao=7, accuracy=1e-4)
    f1, t1, e1 = _forces_torques_energy(s)
    f2, t2, e2 = _forces_torques_energy(s)
    assert np.array_equal(f1, f2) and np.array_equal(t1, t2) and e1 == e2


def _madelung(case, pos, dips):
    k = MAG[case]
    n, sp, dipm = k["n_part"], k["spacing"], MAG["dipm"]
    s = _system(n * sp, pos * sp, dipm * np.asarray(dips, dtype=float))
    s.magnetostatics.solver = DipolarP3M(prefactor=1.0, accuracy=k["accuracy"], mesh=k["mesh"],
                                         cao=k["cao"], r_cut=k["r_cut"], alpha=k["alpha"],
                                         tune=False)
    e = s.analysis.energy()["dipolar"]
    return e / len(pos) / dipm ** 2 * sp ** 3


def test_magnetic_wire():
    """p3m_madelung.py: infinite wire of point dipoles, parallel (-2 zeta(3))
    and antiparallel (3/2 zeta(3)) orderings."""
    n = MAG["wire"]["n_part"]
    pos = np.array([[j, 0, 0] for j in range(n)], dtype=float)
    rtol = MAG["wire"]["rtol"]
    np.testing.assert_allclose(_madelung("wire", pos, [[1.0, 0, 0]] * n), -2.0 * zeta(3),
                               rtol=rtol, atol=0)
    np.testing.assert_allclose(_madelung("wire", pos, [[(-1.0) ** j, 0, 0] for j in range(n)]),
                               1.5 * zeta(3), rtol=rtol, atol=0)


def test_magnetic_sheet():
    n = MAG["sheet"]["n_part"]
    pos, par, anti = [], [], []
    for j, k in itertools.product(range(n), repeat=2):
        th = (-1) ** k * np.pi / 4 + np.pi if j % 2 == 0 else (-1) ** (k + 1) * np.pi / 4
        anti.append([np.cos(th), np.sin(th), 0.0])
        par.append([0.0, (-1.0) ** j, 0.0])
        pos.append([j, k, 0])
    pos = np.array(pos, dtype=float)
    rtol = MAG["sheet"]["rtol"]
    np.testing.assert_allclose(_madelung("sheet", pos, par), MAG["sheet"]["parallel"], rtol=rtol,
                               atol=0)
    np.testing.assert_allclose(_madelung("sheet", pos, anti), MAG["sheet"]["antiparallel"],
                               rtol=rtol, atol=0)


def test_magnetic_cube():
    n = MAG["cube"]["n_part"]
    pos, par, anti = [], [], []
    for i, j, k in itertools.product(range(n), repeat=3):
        th = np.pi + (-1) ** j * np.pi / 4 if i % 2 == 0 else (-1) ** (j + 1) * np.pi / 4
        anti.append([np.cos(th), np.sin(th), 0.0])
        par.append([0.0, 0.0, (-1.0) ** (i + j)])
        pos.append([i, j, k])
    pos = np.array(pos, dtype=float)
    np.testing.assert_allclose(_madelung("cube", pos, par), MAG["cube"]["parallel"],
                               rtol=MAG["cube"]["rtol"], atol=0)
    np.testing.assert_allclose(_madelung("cube", pos, anti), MAG["cube"]["antiparallel"],
                               rtol=MAG["cube"]["rtol_antiparallel"], atol=0)


def _verr(a, b):
    return np.sum(np.linalg.norm(a - b, axis=1)) / np.sqrt(len(a))


def test_golden_1000_dipoles_fixed_parameters():
    """dipolar_mdlc_p3m_scafacos_p2nfft.py:115-152: 1000 dipoles, prefactor
    1.1, mesh 32: energy to 1e-3, forces and torques to 2e-3; and the oracle
    to FP64 rounding."""
    g = np.load(os.path.join(GOLD, "p3m_magnetostatics.npz"))
    L, pref = float(g["box"]), float(g["prefactor"])
    s = _system(L, g["pos"], g["dip"])
    s.magnetostatics.solver = DipolarP3M(prefactor=pref, accuracy=float(g["accuracy"]),
                                         mesh=int(g["mesh"]), cao=7, alpha=0.35, r_cut=10.0,
                                         tune=False)
    f, t, e = _forces_torques_energy(s)
    assert abs(e - float(g["energy"]) * pref) < float(g["energy_tol"])
    assert _verr(f, g["forces"] * pref) < float(g["force_tol"])
    assert _verr(t, g["torques"] * pref) < float(g["torque_tol"])
    fo, to, eo = O.dp3m(L, g["pos"], g["dip"], pref, 0.35, 10.0, int(g["mesh"]), 7,
                        float(g["accuracy"]))
    assert _rel(f, fo) < 1e-9 and _rel(t, to) < 1e-9
    assert e == pytest.approx(eo, rel=1e-10)


def test_golden_1000_dipoles_tuned():
    """dipolar_mdlc_p3m_scafacos_p2nfft.py:133-152 as written: mesh 32,
    accuracy 1e-6, epsilon 'metallic', cao, r_cut and alpha from the tuner
    (DipolarTuningAlgorithm); the achieved estimate meets the target and the
    result the test's tolerances."""
    g = np.load(os.path.join(GOLD, "p3m_magnetostatics.npz"))
    L, pref = float(g["box"]), float(g["prefactor"])
    s = _system(L, g["pos"], g["dip"])
    act = DipolarP3M(prefactor=pref, mesh=int(g["mesh"]), accuracy=float(g["accuracy"]),
                     epsilon="metallic", verbose=False)
    s.magnetostatics.solver = act
    p = act.get_params()
    assert p["is_tuned"] and p["accuracy"] <= float(g["accuracy"])
    assert p["mesh"] == [32, 32, 32] and 1 <= p["cao"] <= 7
    f, t, e = _forces_torques_energy(s)
    assert abs(e - float(g["energy"]) * pref) < float(g["energy_tol"])
    assert _verr(f, g["forces"] * pref) < float(g["force_tol"])
    assert _verr(t, g["torques"] * pref) < float(g["torque_tol"])


def test_tuner_chooses_the_mesh_too():
    """All four parameters tuned for accuracy 1e-4: the estimate meets the
    target, and the rms force error against the converged golden forces
    stays within 3x the target (the estimate is statistical)."""
    g = np.load(os.path.join(GOLD, "p3m_magnetostatics.npz"))
    L, pref = float(g["box"]), float(g["prefactor"])
    s = _system(L, g["pos"], g["dip"])
    act = DipolarP3M(prefactor=pref, accuracy=1e-4, verbose=False)
    s.magnetostatics.solver = act
    p = act.get_params()
    assert p["is_tuned"] and p["accuracy"] <= 1e-4
    f, t, _ = _forces_torques_energy(s)
    ferr = np.sqrt(((f - g["forces"] * pref) ** 2).sum(1).mean())
    assert ferr < 3e-4, (ferr, p)


def test_tuning_needs_dipoles_and_checks_geometry():
    s = _system(10.0, np.zeros((2, 3)), np.zeros((2, 3)))
    with pytest.raises(Exception, match="no dipolar particles"):
        s.magnetostatics.solver = DipolarP3M(prefactor=1.0, accuracy=1e-4)
    assert s.magnetostatics.solver is None
    s2 = eb.System(box_l=[10.0, 10.0, 12.0])
    s2.time_step = 0.01
    s2.part.add(pos=np.ones((2, 3)), dip=np.ones((2, 3)))
    with pytest.raises(Exception, match="requires a cubic box"):
        s2.magnetostatics.solver = DipolarP3M(prefactor=1.0, accuracy=1e-4, mesh=16, cao=3,
                                              alpha=1.0, r_cut=2.0, tune=False)


def test_md_run_with_dipolar_forces():
    """A short velocity-Verlet run: the dipolar forces enter the integrator
    (translations), and the particle count can change between calls."""
    L, n = 10.0, 40
    pos, dip = _random(n, L, 8)
    s = _system(L, pos, dip)
    s.magnetostatics.solver = DipolarP3M(prefactor=1.0, tune=False, alpha=0.9, r_cut=3.0,
                                         mesh=16, cao=5, accuracy=1e-4)
    s.integrator.run(5)
    assert np.all(np.isfinite(s.part.all().pos))
    s.part.add(pos=[1.0, 2.0, 3.0], dip=[0.5, 0.0, 0.0])
    f, t, e = _forces_torques_energy(s)
    fo, to, eo = O.dp3m(L, s.part.all().pos, s.part.all().dip, 1.0, 0.9, 3.0, 16, 5, 1e-4)
    assert _rel(f, fo) < 1e-9 and _rel(t, to) < 1e-9


def test_c_abi_device_pointers_and_energy_only():
    """p3mx_dp3m_compute through the C ABI with device pointers (torch CUDA
    tensors), accumulating into given forces and torques (no
    P3MX_OVERWRITE), and an energy-only call, against the host-pointer
    results of the same handle."""
    import ctypes
    import torch
    from espresso_b200 import _lib
    L, n = 10.0, 70
    pos, dip = _random(n, L, 31)
    act = DipolarP3M(prefactor=1.2, tune=False, alpha=0.9, r_cut=3.0, mesh=16, cao=5,
                     accuracy=1e-4)
    act._set_system([L] * 3, 0.4, (True,) * 3)
    act._activate(pos, dip)
    f_h, t_h, e_h = act._compute(pos, dip, forces=True, energy=True)
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    pos_d = torch.from_numpy(pos).to(dev)
    dip_d = torch.from_numpy(dip).to(dev)
    f0 = torch.full((n, 3), 0.5, dtype=torch.float64, device=dev)
    t0 = torch.full((n, 3), -0.25, dtype=torch.float64, device=dev)
    e = np.zeros(2)
    flags = _lib.P3MX_DEVICE_PTRS | _lib.P3MX_FORCES | _lib.P3MX_ENERGY
    rc = lib.p3mx_dp3m_compute(act._handle, n, _lib.dptr(pos_d), _lib.dptr(dip_d), _lib.dptr(f0),
                               _lib.dptr(t0), e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                               flags, None)
    act._check(rc)
    torch.cuda.synchronize(dev)
    # the same kernels on the same inputs: equal up to the rounding of the
    # offsets the results were added to
    assert _rel(f0.cpu().numpy() - 0.5, f_h) < 1e-12
    assert _rel(t0.cpu().numpy() + 0.25, t_h) < 1e-12
    assert e.sum() == pytest.approx(e_h, rel=1e-13)
    _, _, e_only = act._compute(pos, dip, forces=False, energy=True)
    assert e_only == pytest.approx(e_h, rel=1e-13)
    count = ctypes.c_longlong()
    act._check(lib.p3mx_dp3m_launch_count(act._handle, ctypes.byref(count)))
    assert count.value > 0


def test_stage_profile_entry_point():
    import ctypes
    from espresso_b200 import _lib
    L, n = 10.0, 50
    pos, dip = _random(n, L, 32)
    act = DipolarP3M(prefactor=1.0, tune=False, alpha=0.9, r_cut=3.0, mesh=16, cao=5,
                     accuracy=1e-4)
    act._set_system([L] * 3, 0.4, (True,) * 3)
    act._activate(pos, dip)
    lib = _lib.load()
    names = (ctypes.c_char_p * 32)()
    ms = (ctypes.c_double * 32)()
    nst = ctypes.c_int()
    p = _lib.as_f64(pos)
    d = _lib.as_f64(dip)
    act._check(lib.p3mx_dp3m_profile(act._handle, n, _lib.dptr(p), _lib.dptr(d), 2, ms, names, 32,
                                     ctypes.byref(nst)))
    got = {names[k].decode() for k in range(nst.value)}
    assert {"dp_assign_fft_z", "dp_x_pass", "dp_interp", "dp_pairs"} <= got
    assert all(ms[k] >= 0.0 for k in range(nst.value))
