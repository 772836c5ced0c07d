"""Shared builders for the reference's golden systems (test helpers)."""
import itertools
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def known():
    with open(os.path.join(GOLDEN, "known_answers.json")) as fh:
        return json.load(fh)


def madelung_system(kind):
    """Ionic wire / sheet / cube lattices of p3m_madelung.py:202-313."""
    ka = known()["madelung_" + kind]
    n = ka["n_pairs"]
    pos, q = [], []
    if kind == "wire":
        box = [n / 2, n / 2, 2 * n]
        for i in range(n):
            pos += [[0., 0., 2. * i], [0., 0., 2. * i + 1.]]
            q += [1., -1.]
    elif kind == "sheet":
        box = [2 * n, 2 * n, 4 * n]
        for j, k in itertools.product(range(2 * n), repeat=2):
            pos.append([j, k, 0.])
            q.append((-1.) ** (j + k))
    else:
        box = [2 * n] * 3
        for j, k, l in itertools.product(range(2 * n), repeat=3):
            pos.append([j, k, l])
            q.append((-1.) ** (j + k + l))
    return (np.array(box, float), np.array(pos, float), np.array(q, float), ka)


def jittered_lattice(n_side, box, jitter, seed, valence=1.0):
    """Alternating +/- charges on a jittered simple-cubic lattice."""
    rng = np.random.default_rng(seed)
    a = box / n_side
    idx = np.array(list(itertools.product(range(n_side), repeat=3)), float)
    pos = (idx + 0.5) * a + rng.uniform(-jitter, jitter, idx.shape)
    q = np.where(idx.sum(1) % 2 == 0, valence, -valence)
    return pos, q


def c1_system(seed=0, n=2000, box=20.0, jitter=0.2):
    """The 2000-charge system of the CPU-runnable configuration: a jittered
    simple-cubic lattice of side 13 in a box of side 20 with alternating
    charges, thinned symmetrically to n/2 ions of each sign."""
    side = int(np.ceil(n ** (1.0 / 3.0)))
    rng = np.random.default_rng(seed)
    a = box / side
    idx = np.array(list(itertools.product(range(side), repeat=3)), float)
    q = np.where(idx.sum(1) % 2 == 0, 1.0, -1.0)
    pos = (idx + 0.5) * a + rng.uniform(-jitter, jitter, idx.shape)
    plus, minus = np.flatnonzero(q > 0), np.flatnonzero(q < 0)
    keep = np.zeros(len(q), bool)
    keep[rng.choice(plus, n // 2, replace=False)] = True
    keep[rng.choice(minus, n // 2, replace=False)] = True
    return pos[keep].copy(), q[keep].copy(), box
