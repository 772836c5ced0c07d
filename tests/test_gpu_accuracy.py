"""Accuracy of the headline workload at full size against the FP64 direct
Ewald sum.

The workload is the one the throughput metric is quoted on: 2^20 ions (half
+1, half -1) at density 0.5 in a box of side 128 on a jittered lattice, P3M
with mesh 256^3, cao 7, r_cut 3.5 and alpha from the accuracy formula of
p3m.cpp:636-655 for a target of 1e-4.  Coulomb forces (no LJ) of the
FP32-mixed (P3MGPU) and the plain FP64 (P3M) GPU paths, and of the oracle's
CPU P3M, are compared on a seeded subsample of 20 000 ions with the Ewald
forces that all 2^20 sources exert on them (oracle.ewald_targets, alpha 0.15,
r_cut 27, |n| <= 30: truncation terms exp(-16) and exp(-24)).  The metric is
quoted at an rms force error <= 1e-4.
"""
import numpy as np
import pytest

import bench
import espresso_b200 as eb
from espresso_b200.electrostatics import P3M, P3MGPU
from oracle import oracle as O

pytestmark = pytest.mark.gpu

N_SUB = 20000
EWALD = dict(alpha=0.15, r_cut=27.0, kmax=30)


@pytest.fixture(scope="module")
def headline():
    pos, q, box = bench.make_workload(seed=0, box=128.0)
    args = type("A", (), dict(r_cut=3.5, accuracy=1e-4))()
    alpha = bench.tuned_alpha(args, len(q), float(np.sum(q * q)), box)
    sub = np.sort(np.random.default_rng(2024).choice(len(q), N_SUB, replace=False))
    fe = O.ewald_targets([box] * 3, pos, q, sub, 1.0, **EWALD)
    return pos, q, box, alpha, sub, fe


def _rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum(1).mean()))


@pytest.mark.parametrize("cls", [P3MGPU, P3M])
def test_full_size_rms_force_error_vs_ewald(headline, cls):
    pos, q, box, alpha, sub, fe = headline
    s = eb.System(box_l=[box] * 3)
    s.time_step = 0.01
    s.cell_system.skin = 0.4
    s.part.add(pos=pos, q=q)
    s.electrostatics.solver = cls(prefactor=1.0, accuracy=1e-4, mesh=256, cao=7, r_cut=3.5,
                                  alpha=alpha, tune=False)
    s.integrator.run(0)
    f = s.part.all().f[sub]
    err = _rms(f, fe)
    # the measured error sits at the estimate's level (7.9e-5), not far below
    # it: the comparison resolves the P3M discretisation error
    assert 1e-5 < err <= 1e-4, err


def test_oracle_p3m_on_the_same_subsample(headline):
    """The oracle's CPU P3M (the reference's algorithm in FP64) on the same
    configuration: its error against Ewald is the P3M discretisation error
    the GPU paths must reproduce."""
    pos, q, box, alpha, sub, fe = headline
    p = O.make_params(box, 256, 7, alpha, 3.5, 1.0)
    fk, _, _ = O.p3m_kspace(p, pos, q)
    fr, _, _, _ = O.short_range(p, pos, q)
    err = _rms((fk + fr)[sub], fe)
    assert 1e-5 < err <= 1e-4, err
