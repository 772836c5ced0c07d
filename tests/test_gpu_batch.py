"""GPU tests of the batched-replica API (p3mx_batch_*): many independent
systems of uneven size, box and Bjerrum length advanced by one launch per
kernel.  Forces of every replica are checked against the FP64 oracle with the
parameters the batch autotuner chose; the graph-captured Langevin run is
checked for reproducibility and equipartition.
"""
import ctypes

import numpy as np
import pytest

from espresso_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu

_P = ctypes.POINTER


def make_replicas(seed=5, n_rep=5):
    rng = np.random.default_rng(seed)
    boxes, prefs, pos, q, offs = [], [], [], [], [0]
    for r in range(n_rep):
        n = int(rng.integers(200, 900)) * 2
        L = (n / 0.3) ** (1 / 3)
        nval = n // 2
        val = rng.choice([1.0, 2.0])
        qq = np.concatenate([np.full(nval, val), np.full(nval, -val)])
        # keep ions apart: jittered lattice with random assignment of charges
        side = int(np.ceil(n ** (1 / 3)))
        grid = np.stack(np.meshgrid(*[np.arange(side)] * 3, indexing="ij"), -1).reshape(-1, 3)
        sel = rng.choice(len(grid), n, replace=False)
        p = (grid[sel] + 0.5) * (L / side) + rng.uniform(-0.1, 0.1, (n, 3))
        rng.shuffle(qq)
        boxes.append([L, L, L])
        prefs.append(float(rng.uniform(0.5, 4.0)))
        pos.append(p)
        q.append(qq)
        offs.append(offs[-1] + n)
    return (np.array(boxes), np.array(prefs), np.vstack(pos), np.concatenate(q),
            np.array(offs, dtype=np.int64))


def wca_table():
    tab = (_lib.PairParams * 1)()
    tab[0].wca_eps = 1.0
    tab[0].wca_sig = 1.0
    return tab


def create(boxes, prefs, pos, q, offs, acc=1e-3, single=1, cao=(3, 7)):
    lib = _lib.load()
    d = _lib.BatchDesc()
    d.n_rep = len(prefs)
    boxes = np.ascontiguousarray(boxes, dtype=np.float64)
    prefs = np.ascontiguousarray(prefs, dtype=np.float64)
    offs = np.ascontiguousarray(offs, dtype=np.int64)
    d.box = boxes.ctypes.data_as(_P(ctypes.c_double))
    d.prefactor = prefs.ctypes.data_as(_P(ctypes.c_double))
    d.offset = offs.ctypes.data_as(_P(ctypes.c_longlong))
    d.accuracy = acc
    d.skin = 0.4
    d.single_precision = single
    d.mesh_min, d.mesh_max = 8, 32
    d.cao_min, d.cao_max = cao
    h = ctypes.c_void_p()
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    types = np.zeros(len(q), dtype=np.int32)
    rc = lib.p3mx_batch_create(ctypes.byref(d), pos.ctypes.data_as(_P(ctypes.c_double)),
                               q.ctypes.data_as(_P(ctypes.c_double)),
                               types.ctypes.data_as(_P(ctypes.c_int)), 1, wca_table(),
                               ctypes.byref(h))
    if rc:
        msg = lib.p3mx_batch_last_error(h).decode() if h.value else ""
        raise RuntimeError(f"batch create failed {rc}: {msg}")
    # keep the arrays referenced by the descriptor alive for the call only
    return h


def tuned(h, r):
    t = _lib.Tuned()
    assert _lib.load().p3mx_batch_get_tuned(h, r, ctypes.byref(t)) == 0
    return t


def test_batch_forces_match_oracle_per_replica():
    lib = _lib.load()
    boxes, prefs, pos, q, offs = make_replicas()
    h = create(boxes, prefs, pos, q, offs)
    try:
        R = len(prefs)
        en = np.zeros(R)
        assert lib.p3mx_batch_forces(h, en.ctypes.data_as(_P(ctypes.c_double))) == 0
        f = np.zeros_like(pos)
        assert lib.p3mx_batch_get(h, None, f.ctypes.data_as(_P(ctypes.c_double)), None) == 0
        tab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
        for r in range(R):
            t = tuned(h, r)
            assert t.accuracy <= 1e-3
            sl = slice(offs[r], offs[r + 1])
            p = O.make_params(boxes[r], list(t.mesh), t.cao, t.alpha, t.r_cut, prefs[r])
            fk, ek, _ = O.p3m_kspace(p, pos[sl], q[sl])
            fr, er, _, _ = O.short_range(p, pos[sl], q[sl], None, 1, tab)
            ref = fk + fr
            scale = np.abs(ref).max()
            np.testing.assert_allclose(f[sl], ref, atol=3e-5 * scale, rtol=0)
            e_ref = ek + er[0] + er[1]
            assert abs(en[r] - e_ref) <= 1e-4 * (abs(e_ref) + np.abs(ek) + 1.0)
    finally:
        lib.p3mx_batch_destroy(h)


def test_batch_per_replica_cao_matches_oracle():
    """Replicas of one batch with different charge-assignment orders
    (p3mx_batch_set_cao: each replica takes the tuner's mesh, r_cut and
    alpha for its order): forces and energies of every replica against the
    FP64 oracle, then a graph-captured Langevin run and the forces again."""
    lib = _lib.load()
    boxes, prefs, pos, q, offs = make_replicas(seed=13, n_rep=5)
    h = create(boxes, prefs, pos, q, offs, cao=(3, 7))
    try:
        R = len(prefs)
        want = np.array([5, 7, 6, 7, 5], dtype=np.int32)
        rc = lib.p3mx_batch_set_cao(h, want.ctypes.data_as(_P(ctypes.c_int)))
        assert rc == 0, lib.p3mx_batch_last_error(h).decode()
        bad = np.array([2, 7, 6, 7, 5], dtype=np.int32)
        assert lib.p3mx_batch_set_cao(h, bad.ctypes.data_as(_P(ctypes.c_int))) != 0
        tab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
        for stage in range(2):
            if stage == 1:
                assert lib.p3mx_batch_run(h, 20, 0.005, 1.0, 1.0, 3) == 0
            en = np.zeros(R)
            assert lib.p3mx_batch_forces(h, en.ctypes.data_as(_P(ctypes.c_double))) == 0
            x = np.zeros_like(pos)
            f = np.zeros_like(pos)
            assert lib.p3mx_batch_get(h, x.ctypes.data_as(_P(ctypes.c_double)),
                                      f.ctypes.data_as(_P(ctypes.c_double)), None) == 0
            for r in range(R):
                t = tuned(h, r)
                assert t.cao == want[r]
                assert t.accuracy <= 1e-3
                sl = slice(offs[r], offs[r + 1])
                p = O.make_params(boxes[r], list(t.mesh), t.cao, t.alpha, t.r_cut, prefs[r])
                fk, ek, _ = O.p3m_kspace(p, x[sl], q[sl])
                fr, er, _, _ = O.short_range(p, x[sl], q[sl], None, 1, tab)
                ref = fk + fr
                np.testing.assert_allclose(f[sl], ref, atol=3e-5 * np.abs(ref).max(), rtol=0)
                e_ref = ek + er[0] + er[1]
                assert abs(en[r] - e_ref) <= 1e-4 * (abs(e_ref) + np.abs(ek) + 1.0)
    finally:
        lib.p3mx_batch_destroy(h)


def test_batch_langevin_run_is_reproducible_and_thermalises():
    lib = _lib.load()
    boxes, prefs, pos, q, offs = make_replicas(seed=9, n_rep=3)
    outs = []
    # the autotuner times trials to pick cao; fix cao so both batches get the
    # same parameters (the mesh choice per replica is then deterministic)
    for _ in range(2):
        h = create(boxes, prefs, pos, q, offs, cao=(5, 5))
        try:
            assert lib.p3mx_batch_run(h, 400, 0.005, 1.0, 1.0, 1234) == 0
            x = np.zeros_like(pos)
            v = np.zeros_like(pos)
            assert lib.p3mx_batch_get(h, x.ctypes.data_as(_P(ctypes.c_double)), None,
                                      v.ctypes.data_as(_P(ctypes.c_double))) == 0
            outs.append((x, v))
        finally:
            lib.p3mx_batch_destroy(h)
    # same seed and inputs: bitwise identical trajectories
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    x, v = outs[0]
    assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
    # equipartition within sampling noise: <v^2> per component ~ kT
    assert 0.8 < np.mean(v ** 2) < 1.2


def test_batch_rejects_bad_descriptors():
    lib = _lib.load()
    boxes, prefs, pos, q, offs = make_replicas(n_rep=2)
    with pytest.raises(RuntimeError, match="prefactor"):
        create(boxes, -prefs, pos, q, offs)
    bad = boxes.copy()
    bad[0, 1] *= 1.1
    with pytest.raises(RuntimeError, match="cubic"):
        create(bad, prefs, pos, q, offs)
    del lib


def test_batch_forces_after_langevin_run_match_oracle():
    """After 60 graph-captured Langevin steps (device-side Verlet rebuilds,
    particles crossing cell and box boundaries), a force evaluation at the
    current positions matches the FP64 oracle per replica."""
    lib = _lib.load()
    boxes, prefs, pos, q, offs = make_replicas(seed=13, n_rep=4)
    h = create(boxes, prefs, pos, q, offs, cao=(5, 5))
    try:
        assert lib.p3mx_batch_run(h, 60, 0.005, 1.0, 1.0, 99) == 0
        R = len(prefs)
        en = np.zeros(R)
        assert lib.p3mx_batch_forces(h, en.ctypes.data_as(_P(ctypes.c_double))) == 0
        x = np.zeros_like(pos)
        f = np.zeros_like(pos)
        assert lib.p3mx_batch_get(h, x.ctypes.data_as(_P(ctypes.c_double)),
                                  f.ctypes.data_as(_P(ctypes.c_double)), None) == 0
        assert np.abs(x - pos).max() > 0.05  # the particles did move
        tab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
        for r in range(R):
            t = tuned(h, r)
            sl = slice(offs[r], offs[r + 1])
            p = O.make_params(boxes[r], list(t.mesh), t.cao, t.alpha, t.r_cut, prefs[r])
            fk, _, _ = O.p3m_kspace(p, x[sl], q[sl])
            fr, _, _, _ = O.short_range(p, x[sl], q[sl], None, 1, tab)
            ref = fk + fr
            np.testing.assert_allclose(f[sl], ref, atol=3e-5 * np.abs(ref).max(), rtol=0)
    finally:
        lib.p3mx_batch_destroy(h)


def _nearest_bonds(pos, offs, boxes):
    """One bond per particle of the first half of every replica, to its
    nearest neighbour in the replica (minimum image); global indices."""
    out = []
    for r in range(len(offs) - 1):
        a, b = int(offs[r]), int(offs[r + 1])
        p = pos[a:b]
        L = boxes[r]
        for i in range((b - a) // 2):
            d = p - p[i]
            d -= np.rint(d / L) * L
            d2 = (d * d).sum(1)
            d2[i] = np.inf
            out.append((0, a + i, a + int(np.argmin(d2))))
    return np.array(out, dtype=np.int32)


def test_batch_bonds_in_the_graph_step_match_oracle():
    """FENE bonds inside every replica: p3mx_batch_set_bonds, 40 graph-captured
    Langevin steps, then forces and per-replica energies (bonded included)
    against the FP64 oracle; a bond across replicas is rejected."""
    lib = _lib.load()
    boxes, prefs, pos, q, offs = make_replicas(seed=21, n_rep=3)
    h = create(boxes, prefs, pos, q, offs, cao=(5, 5))
    try:
        bonds = _nearest_bonds(pos, offs, boxes)
        kf, drmax = 10.0, 2.5
        types = (_lib.BondParams * 1)()
        types[0] = _lib.BondParams(_lib.P3MX_BOND_FENE, kf, 0.0, drmax)
        bad = np.array([0, int(offs[0]), int(offs[1])], dtype=np.int32)
        assert lib.p3mx_batch_set_bonds(h, 1, types, 1, bad.ctypes.data_as(_P(ctypes.c_int))) != 0
        assert lib.p3mx_batch_set_bonds(h, 1, types, len(bonds),
                                        bonds.ctypes.data_as(_P(ctypes.c_int))) == 0
        assert lib.p3mx_batch_run(h, 40, 0.005, 1.0, 1.0, 7) == 0
        R = len(prefs)
        en = np.zeros(R)
        assert lib.p3mx_batch_forces(h, en.ctypes.data_as(_P(ctypes.c_double))) == 0
        x = np.zeros_like(pos)
        f = np.zeros_like(pos)
        assert lib.p3mx_batch_get(h, x.ctypes.data_as(_P(ctypes.c_double)),
                                  f.ctypes.data_as(_P(ctypes.c_double)), None) == 0
        assert np.abs(x - pos).max() > 0.05
        tab = O.pair_table(1, {(0, 0): dict(wca_eps=1.0, wca_sig=1.0)})
        for r in range(R):
            t = tuned(h, r)
            a, b = int(offs[r]), int(offs[r + 1])
            sl = slice(a, b)
            mine = bonds[(bonds[:, 1] >= a) & (bonds[:, 1] < b)].copy()
            mine[:, 1:] -= a
            p = O.make_params(boxes[r], list(t.mesh), t.cao, t.alpha, t.r_cut, prefs[r])
            fk, ek, _ = O.p3m_kspace(p, x[sl], q[sl])
            fr, er, _, _ = O.short_range(p, x[sl], q[sl], None, 1, tab)
            fb, eb, _ = O.bonds(boxes[r], x[sl], [(O.BOND_FENE, kf, 0.0, drmax)], mine)
            ref = fk + fr + fb
            np.testing.assert_allclose(f[sl], ref, atol=3e-5 * np.abs(ref).max(), rtol=0)
            e_ref = ek + er[0] + er[1] + eb
            assert abs(en[r] - e_ref) <= 1e-4 * (abs(e_ref) + np.abs(ek) + 1.0)
    finally:
        lib.p3mx_batch_destroy(h)
