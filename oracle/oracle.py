"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the FP64 CPU oracle.

The oracle restates the reference (ESPResSo) CPU P3M + short-range path in
FP64 and adds an independent direct Ewald sum.  Only the test suite, the
smoke check and the CPU-baseline leg of bench.py import this module; the
product path never does.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_REF = os.path.join(_HERE, "_ref", "libref_math.so")


class P3MParams(ctypes.Structure):
    _fields_ = [("box", ctypes.c_double * 3), ("mesh", ctypes.c_int * 3),
                ("cao", ctypes.c_int), ("alpha", ctypes.c_double),
                ("r_cut", ctypes.c_double), ("prefactor", ctypes.c_double),
                ("epsilon", ctypes.c_double), ("mesh_off", ctypes.c_double * 3),
                ("skin", ctypes.c_double)]


class PairParams(ctypes.Structure):
    _fields_ = [("lj_eps", ctypes.c_double), ("lj_sig", ctypes.c_double),
                ("lj_cut", ctypes.c_double), ("lj_shift", ctypes.c_double),
                ("lj_offset", ctypes.c_double), ("lj_min", ctypes.c_double),
                ("wca_eps", ctypes.c_double), ("wca_sig", ctypes.c_double)]


def build():
    """Compile liboracle.so (and the reference-math shim when the reference
    tree is present) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _load():
    if not os.path.exists(_LIB):
        build()
    lib = ctypes.CDLL(_LIB)
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    lp = ctypes.POINTER(ctypes.c_long)
    pp = ctypes.POINTER(P3MParams)
    lib.oracle_p3m_kspace.argtypes = [pp, ctypes.c_long, dp, dp, dp, dp, dp, dp]
    lib.oracle_influence_function.argtypes = [pp, dp]
    lib.oracle_short_range.argtypes = [pp, ctypes.c_long, dp, dp, ip, ctypes.c_int,
                                       ctypes.POINTER(PairParams), dp, dp, dp]
    lib.oracle_cell_grid.argtypes = [dp, ctypes.c_double, ip, dp]
    lib.oracle_cell_index.argtypes = [dp, ctypes.c_double, ctypes.c_long, dp, ip]
    lib.oracle_verlet_pairs.argtypes = [dp, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_long, dp, dp, ip, ctypes.c_int,
                                        dp, ctypes.c_long, lp]
    lib.oracle_verlet_pairs.restype = ctypes.c_long
    lib.oracle_rs_error.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double, dp]
    lib.oracle_rs_error.restype = ctypes.c_double
    lib.oracle_ks_error.argtypes = [ctypes.c_double, ip, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double, dp]
    lib.oracle_ks_error.restype = ctypes.c_double
    lib.oracle_ewald.argtypes = [dp, ctypes.c_long, dp, dp, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 ctypes.c_double, dp, dp]
    lib.oracle_ewald_targets.argtypes = [dp, ctypes.c_long, dp, dp, ctypes.c_long, lp,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, dp]
    for name in ("oracle_bspline", "oracle_as_erfc_part", "oracle_sinc",
                 "oracle_cotangent_sum"):
        getattr(lib, name).restype = ctypes.c_double
    lib.oracle_bspline.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    lib.oracle_as_erfc_part.argtypes = [ctypes.c_double]
    lib.oracle_sinc.argtypes = [ctypes.c_double]
    lib.oracle_cotangent_sum.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    return lib


lib = _load()


def ref_math():
    """The reference's own math headers behind a C ABI, or None when the
    shim was not built (reference tree absent)."""
    if not os.path.exists(_REF):
        return None
    r = ctypes.CDLL(_REF)
    for name in ("ref_bspline", "ref_as_erfc_part", "ref_sinc", "ref_cotangent_sum"):
        getattr(r, name).restype = ctypes.c_double
    r.ref_bspline.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    r.ref_as_erfc_part.argtypes = [ctypes.c_double]
    r.ref_sinc.argtypes = [ctypes.c_double]
    r.ref_cotangent_sum.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
    return r


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def make_params(box, mesh, cao, alpha, r_cut, prefactor, epsilon=0.0,
                mesh_off=(0.5, 0.5, 0.5), skin=0.4):
    p = P3MParams()
    box = np.broadcast_to(np.asarray(box, dtype=float), (3,))
    mesh = np.broadcast_to(np.asarray(mesh, dtype=int), (3,))
    for d in range(3):
        p.box[d] = float(box[d])
        p.mesh[d] = int(mesh[d])
        p.mesh_off[d] = float(mesh_off[d])
    p.cao, p.alpha, p.r_cut = int(cao), float(alpha), float(r_cut)
    p.prefactor, p.epsilon, p.skin = float(prefactor), float(epsilon), float(skin)
    return p


def p3m_kspace(params, pos, q, want_mesh=False):
    """k-space forces (N,3), energy and the k-space virial tensor (3,3)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    n = len(q)
    f = np.zeros((n, 3))
    e = np.zeros(1)
    v = np.zeros(9)
    rho = np.zeros(tuple(params.mesh)) if want_mesh else None
    rc = lib.oracle_p3m_kspace(ctypes.byref(params), n, _d(pos), _d(q), _d(f),
                               _d(e), _d(v), _d(rho) if want_mesh else None)
    if rc:
        raise RuntimeError(f"oracle_p3m_kspace failed ({rc})")
    out = (f, e[0], v.reshape(3, 3))
    return out + (rho,) if want_mesh else out


def influence_function(params):
    g = np.zeros(tuple(params.mesh))
    lib.oracle_influence_function(ctypes.byref(params), _d(g))
    return g


def pair_table(ntypes, entries):
    """entries: dict {(ti, tj): dict(lj_eps=..., ...)} filled symmetrically."""
    tab = (PairParams * (ntypes * ntypes))()
    for (a, b), kw in entries.items():
        for (x, y) in ((a, b), (b, a)):
            e = tab[x * ntypes + y]
            for k, v in kw.items():
                setattr(e, k, float(v))
    return tab


def short_range(params, pos, q, types=None, ntypes=1, tab=None):
    """Real-space Coulomb + LJ/WCA forces, energies {coulomb, non_bonded}
    and virials (two 3x3)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    n = len(q)
    f = np.zeros((n, 3))
    e = np.zeros(2)
    v = np.zeros(18)
    t = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
    rc = lib.oracle_short_range(ctypes.byref(params), n, _d(pos), _d(q),
                                _i(t) if t is not None else None, ntypes, tab,
                                _d(f), _d(e), _d(v))
    if rc:
        raise RuntimeError(f"oracle_short_range failed ({rc})")
    return f, e, v[:9].reshape(3, 3), v[9:].reshape(3, 3)


def cell_grid(box, range_):
    box = np.ascontiguousarray(box, dtype=np.float64)
    cg = np.zeros(3, dtype=np.int32)
    cs = np.zeros(3)
    rc = lib.oracle_cell_grid(_d(box), float(range_), _i(cg), _d(cs))
    if rc:
        raise RuntimeError(f"oracle_cell_grid failed ({rc})")
    return cg, cs


def cell_index(box, range_, pos):
    box = np.ascontiguousarray(box, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    out = np.zeros(len(pos), dtype=np.int32)
    rc = lib.oracle_cell_index(_d(box), float(range_), len(pos), _d(pos), _i(out))
    if rc:
        raise RuntimeError(f"oracle_cell_index failed ({rc})")
    return out


def verlet_pairs(box, skin, coulomb_cut, pos, q, types=None, ia_cut=None):
    box = np.ascontiguousarray(box, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    n = len(q)
    if ia_cut is None:
        ia_cut = np.full((1, 1), -1.0)
    ia_cut = np.ascontiguousarray(ia_cut, dtype=np.float64)
    nt = ia_cut.shape[0]
    t = None if types is None else np.ascontiguousarray(types, dtype=np.int32)
    cap = max(16, 64 * n)
    while True:
        out = np.zeros(2 * cap, dtype=np.int64)
        cnt = lib.oracle_verlet_pairs(_d(box), float(skin), float(coulomb_cut), n,
                                      _d(pos), _d(q), _i(t) if t is not None else None,
                                      nt, _d(ia_cut), cap,
                                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_long)))
        if cnt == -1:
            cap *= 4
            continue
        if cnt < 0:
            raise RuntimeError("oracle_verlet_pairs failed")
        return out[:2 * cnt].reshape(-1, 2)


def rs_error(pref, r_cut_iL, n_c_part, sum_q2, alpha_L, box):
    box = np.ascontiguousarray(box, dtype=np.float64)
    return lib.oracle_rs_error(pref, r_cut_iL, n_c_part, sum_q2, alpha_L, _d(box))


def ks_error(pref, mesh, cao, n_c_part, sum_q2, alpha_L, box):
    box = np.ascontiguousarray(box, dtype=np.float64)
    m = np.ascontiguousarray(np.broadcast_to(mesh, (3,)), dtype=np.int32)
    return lib.oracle_ks_error(pref, _i(m), cao, n_c_part, sum_q2, alpha_L, _d(box))


def ewald(box, pos, q, prefactor, alpha, r_cut, kmax, epsilon=0.0):
    box = np.ascontiguousarray(box, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    f = np.zeros((len(q), 3))
    e = np.zeros(1)
    lib.oracle_ewald(_d(box), len(q), _d(pos), _d(q), prefactor, alpha, r_cut,
                     int(kmax), epsilon, _d(f), _d(e))
    return f, e[0]


def ewald_targets(box, pos, q, targets, prefactor, alpha, r_cut, kmax):
    """Direct FP64 Ewald forces (metallic) on the particles `targets` from
    all sources; the real-space cutoff must not exceed half the box."""
    box = np.ascontiguousarray(box, dtype=np.float64)
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    f = np.zeros((len(t), 3))
    rc = lib.oracle_ewald_targets(_d(box), len(q), _d(pos), _d(q), len(t),
                                  t.ctypes.data_as(ctypes.POINTER(ctypes.c_long)),
                                  prefactor, alpha, r_cut, int(kmax), _d(f))
    if rc:
        raise ValueError(f"oracle_ewald_targets failed ({rc})")
    return f


BOND_FENE = 1
BOND_HARMONIC = 2


def bonds(box, pos, bond_types, bond_list):
    """Pair bonds, restated from the reference in FP64 numpy: FENE
    (bonded_interactions/fene.hpp:67-103), harmonic (harmonic.hpp:62-92),
    applied as add_bonded_two_body_force does (forces_inline.hpp:320-350):
    d = get_mi_vector(x_i, x_j) (BoxGeometry.hpp:47-60), F = fac(|d|) d on i,
    -F on j, virial sum F (x) d (pressure.cpp bonded contribution).

    bond_types: list of (kind, k, r0, r_max) with kind BOND_FENE (r_max =
    d_r_max) or BOND_HARMONIC (r_max = r_cut, 0 for none); bond_list: (B, 3)
    ints (type, i, j).  Returns forces (N, 3), energy, virial (3, 3); raises
    RuntimeError("bond broken ...") for a bond past its range and for a
    zero-length bond with r0 > 0, as the reference's runtime errors do.
    """
    box = np.asarray(box, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    bl = np.asarray(bond_list, dtype=np.int64).reshape(-1, 3)
    f = np.zeros_like(pos)
    energy = 0.0
    vir = np.zeros((3, 3))
    for t, i, j in bl:
        kind, k, r0, r_max = bond_types[t]
        d = pos[i] - pos[j]
        far = np.abs(d) > 0.5 * box
        d = np.where(far, d - np.rint(d / box) * box, d)
        ln = np.sqrt(d @ d)
        dr = ln - r0
        if kind == BOND_FENE:
            if dr >= r_max:
                raise RuntimeError("bond broken between particles %d, %d" % (i, j))
            fac = -k * dr / (1.0 - dr * dr / r_max ** 2)
            e = -0.5 * k * r_max ** 2 * np.log(1.0 - dr * dr / r_max ** 2)
        else:
            if r_max > 0.0 and ln > r_max:
                raise RuntimeError("bond broken between particles %d, %d" % (i, j))
            fac = -k * dr
            e = 0.5 * k * dr * dr
        if ln > 1e-14:
            fac /= ln
        elif r0 > 0.0:
            raise RuntimeError("particles %d, %d have zero distance" % (i, j))
        force = fac * d
        f[i] += force
        f[j] -= force
        energy += e
        vir += np.outer(force, d)
    return f, energy, vir


def elc_far_cut(box, box_h, max_pw_error, lz=None):
    """ELC far-formula cutoff from the maximal pairwise error, restating
    ElectrostaticLayerCorrection::tune_far_cut (electrostatics/elc.cpp:942-973):
    lz = L_z, or box_h + space_layer with dielectric contrasts.  Raises
    RuntimeError when no cutoff below 50 meets the bound, as the reference
    does."""
    ux, uy = 1.0 / box[0], 1.0 / box[1]
    umin = min(ux, uy)
    lz = box[2] if lz is None else lz
    fc = umin
    while True:
        pref = 2.0 * np.pi * fc
        s = pref + 2.0 * (ux + uy)
        den = -np.expm1(-pref * lz)
        num1 = np.exp(pref * (box_h - lz))
        num2 = np.exp(-pref * (box_h + lz))
        err = 0.5 / den * (num1 * (s + 1.0 / (lz - box_h)) / (lz - box_h) +
                           num2 * (s + 1.0 / (lz + box_h)) / (lz + box_h))
        fc += umin
        if not (err > max_pw_error and fc < 50.0):
            break
    if fc >= 50.0:
        raise RuntimeError("ELC tuning failed: maxPWerror too small")
    return fc - umin


def elc_modes(box, far_cut):
    """The (p, q) frequencies ELC sums over, in the reference's loop order
    (elc.cpp:830-883): p-modes (q = 0), q-modes (p = 0), then p-major pq
    modes; each as (kind, p, q, omega) with kind 0 = x, 1 = y, 2 = pq."""
    ux, uy = 1.0 / box[0], 1.0 / box[1]
    nfx = int(np.ceil(far_cut * box[0]) + 1.0)
    nfy = int(np.ceil(far_cut * box[1]) + 1.0)
    modes = []
    p = 1
    while ux * (p - 1) < far_cut and p <= nfx:
        modes.append((0, p, 0, 2.0 * np.pi * ux * p))
        p += 1
    q = 1
    while uy * (q - 1) < far_cut and q <= nfy:
        modes.append((1, 0, q, 2.0 * np.pi * uy * q))
        q += 1
    p = 1
    while ux * (p - 1) < far_cut and p <= nfx:
        q = 1
        while (ux * (p - 1)) ** 2 + (uy * (q - 1)) ** 2 < far_cut * far_cut and q <= nfy:
            modes.append((2, p, q, 2.0 * np.pi * np.sqrt((ux * p) ** 2 + (uy * q) ** 2)))
            q += 1
        p += 1
    return modes


def elc(box, gap_size, pos, q, prefactor, far_cut, neutralize=True, delta_top=0.0,
        delta_bot=0.0, const_pot=False, pot_diff=0.0, space_layer=0.0):
    """ELC correction forces and energy in FP64 numpy, restating
    electrostatics/elc.cpp: the dipole force and energy (add_dipole_force
    :201-264, dipole_energy :267-343), the z terms of dielectric contrasts
    (z_energy :366-439, add_z_force :441-494), the per-frequency product
    decomposition with its image-layer terms (setup_PoQ :501-598,
    add_PoQ_force :601-618, PoQ_energy :620-634, setup_PQ :641-769,
    add_PQ_force :771-810, PQ_energy :812-828) and their sums (add_force
    :830-883, calc_energy :885-940, which halves the total).  The flags are
    the effective ones of elc_data (:1056-1102): contrasts switch
    neutralization off and const_pot needs a contrast.  Positions are folded
    into the box first, as the reference's particle positions are.  Returns
    (forces (N, 3), energy); raises RuntimeError for a charged particle in
    the gap.
    """
    box = np.asarray(box, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    pos = pos - np.floor(pos / box) * box
    x, y, z = pos[:, 0], pos[:, 1], pos[:, 2]
    lz = box[2]
    h = lz - gap_size
    contrast = (delta_top != 0.0) or (delta_bot != 0.0)
    const_pot = bool(const_pot) and contrast
    neutralize = bool(neutralize) and not contrast
    pot_diff = pot_diff if const_pot else 0.0
    sl = space_layer if contrast else 0.0
    bad = (q != 0.0) & ((z < 0.0) | (z > h))
    if bad.any():
        i = int(np.flatnonzero(bad)[0])
        dz = z[i] if z[i] < 0.0 else z[i] - h
        raise RuntimeError("Particle %d entered ELC gap region by %r" % (i, dz))
    mb = contrast & (z < sl)
    mt = contrast & (z > h - sl)
    db, dt = delta_bot, delta_top
    f = np.zeros_like(pos)
    vol = box[0] * box[1] * box[2]
    shift = 0.5 * lz
    # dipole force (elc.cpp:201-264)
    pref = prefactor * 4.0 * np.pi / vol
    g0 = np.sum(q * (z - shift)) + np.sum((db * q * (-z - shift))[mb]) + \
        np.sum((dt * q * (2.0 * h - z - shift))[mt])
    g1 = np.sum(q * z)
    g2 = np.sum(q) + np.sum((db * q)[mb]) + np.sum((dt * q)[mt])
    g0 *= pref
    g1 *= pref / h * lz
    g2 *= pref
    field = g0
    if const_pot:
        field -= pot_diff / h + g1
    f[:, 2] -= field * q
    if not neutralize:
        f[:, 2] += g2 * q * (z - shift)
    # dipole energy (elc.cpp:267-343)
    pref = prefactor * 2.0 * np.pi / vol
    s0 = np.sum(q)
    s1 = np.sum((db * q)[mb]) + np.sum((dt * q)[mt])
    s2 = np.sum(q * (z - shift))
    s3 = np.sum((db * q * (-z - shift))[mb]) + np.sum((dt * q * (2.0 * h - z - shift))[mt])
    s4 = np.sum(q * (z - shift) ** 2)
    s5 = np.sum((db * q * (-z - shift) ** 2)[mb]) + \
        np.sum((dt * q * (2.0 * h - z - shift) ** 2)[mt])
    s6 = np.sum(q * z)
    energy = 2.0 * pref * (s2 * s2 + s2 * s3)
    if not neutralize:
        energy += 2.0 * pref * (-s0 * s4 - (0.25 - 0.5 / 3.0) * (s0 * lz) ** 2)
    if contrast:
        if const_pot:
            energy += pref / h * lz * s6 * s6
            energy -= 2.0 * pot_diff / h * s6
        energy += pref * (-(s1 * s4 + s0 * s5) - (1.0 - 2.0 / 3.0) * s0 * s1 * lz * lz)
    area_inv = 1.0 / (box[0] * box[1])
    if contrast:
        # z force and z energy (elc.cpp:366-494)
        pref = prefactor * 2.0 * np.pi * area_inv
        delta = dt * db
        if const_pot:
            gz = np.sum((-db * q)[mb]) + np.sum((dt * q)[mt])
            z2 = gz
            z3 = np.sum((-db * q * (-z - shift))[mb]) + \
                np.sum((dt * q * (2.0 * h - z - shift))[mt])
        else:
            # delta = 1 (two metallic walls) needs const_pot (elc.cpp:1095-1101)
            fdb, fdt, fd = db / (1.0 - delta), dt / (1.0 - delta), delta / (1.0 - delta)
            gz = np.sum(np.where(mb, fd * (db + 1.0) * q, fdb * (dt + 1.0) * q)) - \
                np.sum(np.where(mt, fd * (dt + 1.0) * q, fdt * (db + 1.0) * q))
            dci = 1.0 / (1.0 - delta)

            def img_b(a, zz):
                return a * dci * (zz - 2.0 * delta * lz * dci) - a * dci * shift

            def img_t(a, zz):
                return a * dci * (zz + 2.0 * delta * lz * dci) - a * dci * shift
            z2 = gz
            z3 = np.sum(q * np.where(mb, img_b(db * delta, -(2.0 * h + z)) +
                                     img_b(delta, -(2.0 * h - z)),
                                     img_b(db, -z) + img_b(delta, -(2.0 * h - z))))
            z3 -= np.sum(q * np.where(mt, img_t(dt * delta, 4.0 * h - z) +
                                      img_t(delta, 2.0 * h + z),
                                      img_t(dt, 2.0 * h - z) + img_t(delta, 2.0 * h + z)))
        f[:, 2] += pref * gz * q
        z0 = np.sum(q)
        z1 = np.sum(q * (z - shift))
        energy += -pref * (z1 * z2 - z0 * z3)
    ux, uy = 1.0 / box[0], 1.0 / box[1]
    for kind, p, qq, omega in elc_modes(box, far_cut):
        e = np.exp(omega * z)
        if contrast:
            delta = dt * db
            fac_elc = 1.0 / (1.0 - delta * np.exp(-omega * 2.0 * h))
            fdb, fdt = db * fac_elc, dt * fac_elc
            fd = fdb * dt
            eb = np.exp(-omega * z)
            et = np.exp(omega * (2.0 * h - z))
            e2 = np.where(mb, (np.exp(omega * (-z - 2.0 * h)) * db + np.exp(omega * (z - 2.0 * h))) * fd,
                          (np.exp(-omega * z) + np.exp(omega * (z - 2.0 * h)) * dt) * fdb)
            e3 = np.where(mt, (np.exp(omega * (z - 4.0 * h)) * dt + np.exp(omega * (-z - 2.0 * h))) * fd,
                          (np.exp(omega * (z - 2.0 * h)) + np.exp(omega * (-z - 2.0 * h)) * db) * fdt)
            wb = np.where(mb, q * db, 0.0)
            wt = np.where(mt, q * dt, 0.0)
        if kind < 2:
            c = x if kind == 0 else y
            u = ux if kind == 0 else uy
            arg = (2.0 * np.pi * u * (p if kind == 0 else qq)) * c
            sn, co = np.sin(arg), np.cos(arg)
            pb = np.stack([q * sn * e, q * co * e, q * sn / e, q * co / e])  # SP CP SM CM
            pref_di = prefactor * 4.0 * np.pi * area_inv
            pref = -pref_di / np.expm1(omega * lz)
            gbl = pb.sum(axis=1)
            if contrast:
                gbl = gbl + np.stack([sn * eb, co * eb, sn / eb, co / eb]) @ wb + \
                    np.stack([sn * et, co * et, sn / et, co / et]) @ wt
                lcl = np.array([np.sum(q * sn * e2), np.sum(q * co * e2),
                                np.sum(q * sn * e3), np.sum(q * co * e3)])
                G = pref * gbl + pref_di * lcl
            else:
                G = pref * gbl
            SP, CP, SM, CM = pb
            f[:, kind] += SM * G[1] - CM * G[0] + SP * G[3] - CP * G[2]
            f[:, 2] += CM * G[1] + SM * G[0] - CP * G[3] - SP * G[2]
            energy += np.sum(CM * G[1] + SM * G[0] + CP * G[3] + SP * G[2]) / omega
        else:
            ax = (2.0 * np.pi * ux * p) * x
            ay = (2.0 * np.pi * uy * qq) * y
            sx, cx, sy, cy = np.sin(ax), np.cos(ax), np.sin(ay), np.cos(ay)
            pp = np.stack([sx * sy, sx * cy, cx * sy, cx * cy])  # SS SC CS CC
            pb = np.concatenate([pp * q * e, pp * q / e])
            pref_di = prefactor * 8.0 * np.pi * area_inv
            pref = -pref_di / np.expm1(omega * lz)
            gbl = pb.sum(axis=1)
            if contrast:
                gbl = gbl + np.concatenate([pp * eb, pp / eb]) @ wb + \
                    np.concatenate([pp * et, pp / et]) @ wt
                lcl = np.concatenate([pp @ (q * e2), pp @ (q * e3)])
                G = pref * gbl + pref_di * lcl
            else:
                G = pref * gbl
            SSP, SCP, CSP, CCP, SSM, SCM, CSM, CCM = pb
            px = 2.0 * np.pi * ux * p / omega
            py = 2.0 * np.pi * uy * qq / omega
            f[:, 0] += px * (SCM * G[3] + SSM * G[2] - CCM * G[1] - CSM * G[0] +
                             SCP * G[7] + SSP * G[6] - CCP * G[5] - CSP * G[4])
            f[:, 1] += py * (CSM * G[3] + SSM * G[1] - CCM * G[2] - SCM * G[0] +
                             CSP * G[7] + SSP * G[5] - CCP * G[6] - SCP * G[4])
            f[:, 2] += (CCM * G[3] + CSM * G[2] + SCM * G[1] + SSM * G[0] -
                        CCP * G[7] - CSP * G[6] - SCP * G[5] - SSP * G[4])
            energy += np.sum(CCM * G[3] + CSM * G[2] + SCM * G[1] + SSM * G[0] +
                             CCP * G[7] + CSP * G[6] + SCP * G[5] + SSP * G[4]) / omega
    return f, 0.5 * energy


def _p3m_pair(prefactor, alpha, r_cut, q1q2, d):
    """CoulombP3M::pair_force / pair_energy (electrostatics/p3m.hpp:146-180)
    with the Abramowitz-Stegun erfc part, vectorised over rows of d."""
    d = np.atleast_2d(d)
    q1q2 = np.broadcast_to(np.asarray(q1q2, dtype=np.float64), (len(d),))
    r = np.sqrt(np.sum(d * d, axis=1))
    ok = (q1q2 != 0.0) & (r < r_cut) & (r > 0.0)
    rs = np.where(ok, r, 1.0)
    ad = alpha * rs
    t = 1.0 / (1.0 + 0.3275911 * ad)
    asp = t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 +
                                                                          t * 1.061405429))))
    ex = np.exp(-ad * ad)
    erfc_ri = asp / rs
    fac = ex * (erfc_ri + 2.0 * alpha / np.sqrt(np.pi)) / (rs * rs)
    force = np.where(ok[:, None], (fac * prefactor * q1q2)[:, None] * d, 0.0)
    energy = np.where(ok, prefactor * q1q2 * erfc_ri * ex, 0.0)
    return force, energy


def elc_space_layer(gap_size, box_h, r_cut):
    """recalc_space_layer (elc.cpp:1032-1054): a third of the gap, at most
    gap - r_cut and half the slab; RuntimeError when nothing is left."""
    sl = gap_size / 3.0
    mx = min(gap_size - r_cut, box_h / 2.0)
    if sl > mx:
        if mx <= 0.0:
            raise RuntimeError("P3M real-space cutoff too large for ELC w/ dielectric contrast")
        sl = mx
    return sl


def elc_system(box, gap_size, pos, q, prefactor, alpha, r_cut, mesh, cao, max_pw_error,
               far_cut=-1.0, neutralize=True, delta_top=0.0, delta_bot=0.0,
               const_pot=False, pot_diff=0.0):
    """Coulomb forces and energy of P3M + ELC for the whole system (k-space,
    real space and the correction), restating the reference's combination:
    without contrasts P3M forces and energy plus `elc`; with contrasts
    (ElectrostaticLayerCorrection::add_long_range_forces :1231-1254,
    long_range_energy :1189-1229) the mesh carries the image charges of the
    particles within space_layer of either wall (charge_assign :1111-1142,
    modify_p3m_sums :1144-1187: the P3M sums of that charge set), the
    energy is 0.5 E(real) + 0.5 E(self images) + 0.5 E(real + images)
    - 0.5 E(images), every particle feels its own image
    (dielectric_layers_self_forces, elc.hpp) and every pair the image of
    each partner within space_layer (add_pair_force_corrections /
    pair_energy_correction, elc.hpp: particle 1 gets pair_force(q_eff,
    mi(x2 - image(x1))) and the energy is half the sum over both orders).
    P3M runs metallic (adapt_epsilon_elc).  Returns (forces, energy)."""
    box = np.asarray(box, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64)
    n = len(q)
    h = box[2] - gap_size
    contrast = (delta_top != 0.0) or (delta_bot != 0.0)
    sl = elc_space_layer(gap_size, h, r_cut) if contrast else 0.0
    lz_tune = h + sl if contrast else box[2]
    fc = elc_far_cut(box, h, max_pw_error, lz=lz_tune) if far_cut == -1.0 else far_cut
    prm = make_params(box, mesh, cao, alpha, r_cut, prefactor)
    fr, er, _, _ = short_range(prm, pos, q)
    fe, ee = elc(box, gap_size, pos, q, prefactor, fc, neutralize=neutralize,
                 delta_top=delta_top, delta_bot=delta_bot, const_pot=const_pot,
                 pot_diff=pot_diff, space_layer=sl)
    if not contrast:
        fk, ek, _ = p3m_kspace(prm, pos, q)
        return fk + fr + fe, ek + er[0] + ee
    pf = pos - np.floor(pos / box) * box
    z = pf[:, 2]
    mb = (q != 0.0) & (z < sl)
    mt = (q != 0.0) & (z > h - sl)
    img_b = pf.copy()
    img_b[:, 2] = -z
    img_t = pf.copy()
    img_t[:, 2] = 2.0 * h - z
    ipos = np.concatenate([img_b[mb], img_t[mt]])
    iq = np.concatenate([delta_bot * q[mb], delta_top * q[mt]])
    both_pos = np.concatenate([pf, ipos])
    both_q = np.concatenate([q, iq])
    fk_both, e_both, _ = p3m_kspace(prm, both_pos, both_q)
    _, e_real, _ = p3m_kspace(prm, pf, q)
    _, e_img, _ = p3m_kspace(prm, ipos, iq) if len(iq) else (None, 0.0, None)
    f = fk_both[:n] + fr + fe
    energy = er[0] + ee + 0.5 * e_real + 0.5 * e_both - 0.5 * e_img

    def mi(d):
        return d - np.rint(d / box) * box
    # self images (dielectric_layers_self_forces / _self_energy)
    e_self = 0.0
    for m, img, dl in ((mb, img_b, delta_bot), (mt, img_t, delta_top)):
        idx = np.flatnonzero(m)
        if len(idx):
            fs, es = _p3m_pair(prefactor, alpha, r_cut, dl * q[idx] ** 2, mi(pf[idx] - img[idx]))
            f[idx] += fs
            e_self += es.sum()
    energy += 0.5 * e_self
    # image pairs: particle i in a layer, every partner j != i
    e_pair = 0.0
    for m, img, dl in ((mb, img_b, delta_bot), (mt, img_t, delta_top)):
        for i in np.flatnonzero(m):
            j = np.flatnonzero(np.arange(n) != i)
            fs, es = _p3m_pair(prefactor, alpha, r_cut, dl * q[i] * q[j], mi(pf[j] - img[i]))
            f[i] += fs.sum(axis=0)
            e_pair += es.sum()
    energy += 0.5 * e_pair
    return f, energy


def _meshift(m, zero_mid):
    """detail::calc_meshift (p3m/common.hpp:248-264)."""
    r = np.zeros(m, dtype=np.int64)
    for j in range(1, m // 2 + 1):
        r[j] = j
        r[m - j] = -j
    if zero_mid:
        r[m // 2] = 0
    return r


def _dp3m_influence(M, L, cao, alpha, S):
    """grid_influence_function<S> of the dipolar P3M
    (p3m/influence_function_dipolar.hpp): G_opt_dipolar<S> with m = 0,
    numerator U^2 exp(-pi^2 |n|^2 / alpha_L^2) / |n|^2 (d_op . n)^S,
    denominator |d_op|^(2S) (U^2)^2, zero where all indices are multiples of
    M/2, times 2 M^3 / L^2.  S = 2 for the energy, 3 for the forces.
    Returns (g, keep mask, shift grids, d_op grids)."""
    shift = _meshift(M, False)
    dop = _meshift(M, True)
    sx, sy, sz = np.meshgrid(shift, shift, shift, indexing="ij")
    dx, dy, dz = np.meshgrid(dop, dop, dop, indexing="ij")
    i0, i1, i2 = np.meshgrid(np.arange(M), np.arange(M), np.arange(M), indexing="ij")
    h = M // 2
    keep = (i0 % h != 0) | (i1 % h != 0) | (i2 % h != 0)
    u2 = (np.sinc(sx / M) * np.sinc(sy / M) * np.sinc(sz / M)) ** (2 * cao)
    n2 = (sx * sx + sy * sy + sz * sz).astype(np.float64)
    ex = (np.pi / (alpha * L)) ** 2 * n2
    dn = (dx * sx + dy * sy + dz * sz).astype(np.float64)
    dd = (dx * dx + dy * dy + dz * dz).astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        num = np.where(ex < 30.0, u2 * np.exp(-ex) / n2 * dn ** S, 0.0)
        g = np.where(keep, 2.0 * M ** 3 / L ** 2 * num / (dd ** S * u2 * u2), 0.0)
    return g, keep, (sx, sy, sz), (dx, dy, dz)


def dp3m(box_l, pos, dip, prefactor, alpha, r_cut, mesh, cao, accuracy, want_forces=True,
         epsilon=0.0, mesh_off=(0.5, 0.5, 0.5)):
    """Dipolar P3M (cubic box and mesh, metallic) in FP64 numpy, restating
    magnetostatics/dp3m.cpp and dp3m.hpp: the three dipole-component meshes
    assigned with the charge-assignment weights (dipole_assign; here through
    the charge oracle, one component at a time), the k-space energy
    G_energy |mu(k) . d_op|^2 prefactor pi / (M^3 L) with the self term
    -prefactor sum mu^2 2 alpha^3 / (3 sqrt pi) and the Madelung-self
    correction (long_range_kernel :270-310, calc_energy_correction,
    calc_average_self_energy_k_space with the aliasing sum over
    m in [-1, 1]^3); the k-space torques tau -= mu x (prefactor 2 pi / (M^3 L)
    E), E_d interpolated from the backward transform of
    d_op_d G_energy (mu . d_op) (AssignTorques), and forces
    F_d += mu . (prefactor (2 pi / L)^2 / M^3 E^(d)), E^(d)_c from
    d_op_c d_op_d G_force (-i) (mu . d_op) (AssignForces, :322-420); the
    real-space pair energy, force and torque with B, C, D of dp3m.hpp
    :142-232 over minimum-image pairs within r_cut (exact erfc below accuracy
    5e-6), the partner getting -F and -(tau + d x F) (calc_opposing_force,
    forces_inline.hpp:159-171).  Mesh values are interpolated with each
    particle's own assignment stencil.  For epsilon != 0 the surface term of
    calc_surface_term (dp3m.cpp:452-510): energy + pref/2 |M|^2 and torques
    -pref mu x M, M the total moment, pref = prefactor 4 pi / (V (2 eps + 1)).
    Returns (forces, torques, energy)."""
    L = float(box_l)
    pos = np.asarray(pos, dtype=np.float64)
    dip = np.asarray(dip, dtype=np.float64)
    n = len(pos)
    M = int(mesh)
    prm = make_params([L] * 3, M, cao, alpha, r_cut, 1.0, mesh_off=mesh_off)
    rho = []
    for d in range(3):
        c = np.ascontiguousarray(dip[:, d])
        rho.append(p3m_kspace(prm, pos, c, want_mesh=True)[3] if np.any(c != 0.0)
                   else np.zeros((M, M, M)))
    F = [np.fft.fftn(r) for r in rho]
    g_e, keep, (sx, sy, sz), dops = _dp3m_influence(M, L, cao, alpha, 2)
    mk = F[0] * dops[0] + F[1] * dops[1] + F[2] * dops[2]
    energy = np.sum(g_e * (mk.real ** 2 + mk.imag ** 2)) * prefactor / M ** 3 * np.pi / L
    sum_mu2 = float(np.sum(dip * dip))
    energy -= prefactor * sum_mu2 / np.sqrt(np.pi) * (2.0 / 3.0) * alpha ** 3
    u2s = np.zeros((M, M, M))
    for m0 in (-1, 0, 1):
        for m1 in (-1, 0, 1):
            for m2 in (-1, 0, 1):
                u2s += (np.sinc(sx / M + m0 * M) * np.sinc(sy / M + m1 * M) *
                        np.sinc(sz / M + m2 * M)) ** (2 * cao)
    dd = (dops[0] ** 2 + dops[1] ** 2 + dops[2] ** 2).astype(np.float64)
    phi = np.sum(np.where(keep, g_e * u2s * dd, 0.0))
    vol = L ** 3
    uk = phi / (3.0 * L * M ** 3) * np.pi * vol
    e_self = -2.0 * (alpha * L) ** 3 / np.sqrt(np.pi) / 3.0
    energy += prefactor * (-sum_mu2 * (uk + e_self + 2.0 * np.pi / 3.0)) / vol
    f = np.zeros((n, 3))
    t = np.zeros((n, 3))
    if want_forces and n:
        def back(z):
            return (np.fft.ifftn(z) * M ** 3).real
        e_t = [back(dops[d] * g_e * mk) for d in range(3)]
        g_f = _dp3m_influence(M, L, cao, alpha, 3)[0]
        kf = -1j * g_f * mk
        e_f = [[back(dops[c] * dops[d] * kf) for c in range(3)] for d in range(3)]
        wn = 2.0 * np.pi / L
        pt = prefactor / M ** 3 * wn
        pf = prefactor / M ** 3 * wn * wn
        for i in range(n):
            w = p3m_kspace(prm, pos[i:i + 1], np.ones(1), want_mesh=True)[3]
            nz = np.nonzero(w)
            wv = w[nz]
            et = np.array([wv @ e_t[d][nz] for d in range(3)])
            t[i] -= np.cross(dip[i], pt * et)
            for d in range(3):
                ef = np.array([wv @ e_f[d][c][nz] for c in range(3)])
                f[i, d] += dip[i] @ (pf * ef)
    # real space
    from math import erfc
    coeff = 2.0 * alpha / np.sqrt(np.pi)
    a2 = alpha * alpha
    for i in range(n - 1):
        d = pos[i] - pos[i + 1:]
        d -= np.rint(d / L) * L
        r2 = np.sum(d * d, axis=1)
        r = np.sqrt(r2)
        ok = (r < r_cut) & (r > 0.0)
        if not ok.any():
            continue
        js = np.flatnonzero(ok) + i + 1
        d, r, r2 = d[ok], r[ok], r2[ok]
        mj = dip[js]
        mi = dip[i]
        ad = alpha * r
        exa = np.exp(-ad * ad)
        if accuracy > 5e-6:
            tt = 1.0 / (1.0 + 0.3275911 * ad)
            asp = tt * (0.254829592 + tt * (-0.284496736 + tt * (1.421413741 +
                                                                   tt * (-1.453152027 + tt * 1.061405429))))
            b = (asp / r + coeff) * exa / r2
        else:
            b = (np.array([erfc(x) for x in ad]) / r + coeff * exa) / r2
        common = a2 * coeff * exa
        c = (3.0 * b + 2.0 * common) / r2
        dcoef = (5.0 * c + 4.0 * common * a2) / r2
        mimj = mj @ mi
        mir = d @ mi
        mjr = np.sum(mj * d, axis=1)
        energy += prefactor * np.sum(mimj * b - mir * mjr * c)
        if want_forces:
            fo = prefactor * ((mimj * c)[:, None] * d + np.outer(mjr * c, mi) + mj * (mir * c)[:, None]
                              - (mir * mjr * dcoef)[:, None] * d)
            to = prefactor * (-np.cross(mi, mj) * b[:, None] + np.cross(mi, d) * (mjr * c)[:, None])
            f[i] += fo.sum(axis=0)
            t[i] += to.sum(axis=0)
            f[js] -= fo
            t[js] -= to + np.cross(d, fo)
    if epsilon != 0.0:
        ps = prefactor * 4.0 * np.pi / L ** 3 / (2.0 * epsilon + 1.0)
        mtot = dip.sum(axis=0)
        energy += 0.5 * ps * float(mtot @ mtot)
        t -= ps * np.cross(dip, mtot)
    return f, t, energy


def dp3m_energy(box_l, pos, dip, prefactor, alpha, r_cut, mesh, cao, accuracy):
    """Dipolar P3M energy only (see dp3m)."""
    return dp3m(box_l, pos, dip, prefactor, alpha, r_cut, mesh, cao, accuracy,
                want_forces=False)[2]


def dlc_far_cut(box, box_h, n_magnetic, mu_max, max_pw_error):
    """DipolarLayerCorrection::tune_far_cut (magnetostatics/dlc.cpp:416-460)
    with g1_DLC_dip / g2_DLC_dip (:80-93): the smallest kc < 200 whose error
    estimate is below max_pw_error; RuntimeError otherwise."""
    lx, ly, lz = box
    if abs(lx - ly) > 0.001:
        raise RuntimeError("DLC tuning: box size in x direction is different from y direction."
                           " The tuning formula requires both to be equal.")

    def g1(g, x):
        c = g / x
        x3 = x ** 3
        return g ** 3 / x + 1.5 * c * c + 1.5 * g / x3 + 0.75 / (x3 * x)

    def g2(g, x):
        return g * g / x + 2.0 * g / (x * x) + 2.0 / (x ** 3)
    piarea = np.pi / (lx * ly)
    h = box_h
    for kc in range(1, 200):
        gc = kc * 2.0 * np.pi / lx
        fa0 = np.sqrt(9.0 * np.exp(2.0 * gc * h) * g1(gc, lz - h) +
                      9.0 * np.exp(-2.0 * gc * h) * g1(gc, lz + h) + 22.0 * g1(gc, lz))
        fa1 = np.sqrt(0.125 * piarea) * fa0
        de = n_magnetic * mu_max ** 2 / (4.0 * (np.exp(gc * lz) - 1.0)) * (fa1 + g2(gc, lz))
        if de < max_pw_error:
            return float(kc)
    raise RuntimeError("DLC tuning failed: maxPWerror too small")


def dlc_energy_correction(box, gap_size, pos, dip, prefactor, far_cut):
    """DLC energy correction for a metallic base solver
    (DipolarLayerCorrection::energy_correction, dlc.cpp:356-396, with
    dipolar_energy_correction :247-302 after Brodka): the sum over the
    2D wave vectors |ix|, |iy| <= round(far_cut), (ix, iy) != 0, of
    -pi / (L_x L_y) fa1 2 (S0 S2 + S1 S3) with fa1 = 1 / (g (exp(g L_z) - 1)),
    times the prefactor, plus the shape term prefactor 2 pi / V M_z^2.
    Positions folded; RuntimeError for a magnetic particle in the gap."""
    box = np.asarray(box, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    dip = np.asarray(dip, dtype=np.float64)
    pos = pos - np.floor(pos / box) * box
    mag = np.linalg.norm(dip, axis=1) != 0.0
    h = box[2] - gap_size
    z = pos[:, 2]
    bad = mag & ((z < 0.0) | (z > h))
    if bad.any():
        raise RuntimeError("Particle %d entered DLC gap region" % int(np.flatnonzero(bad)[0]))
    pos, dip = pos[mag], dip[mag]
    kc = int(np.round(far_cut))
    fx, fy = 2.0 * np.pi / box[0], 2.0 * np.pi / box[1]
    e = 0.0
    for ix in range(-kc, kc + 1):
        for iy in range(-kc, kc + 1):
            if ix == 0 and iy == 0:
                continue
            gx, gy = ix * fx, iy * fy
            gr = np.sqrt(gx * gx + gy * gy)
            fa1 = 1.0 / (gr * (np.exp(gr * box[2]) - 1.0))
            a = gx * dip[:, 0] + gy * dip[:, 1]
            b = gr * dip[:, 2]
            er = gx * pos[:, 0] + gy * pos[:, 1]
            c, d = np.cos(er), np.sin(er)
            f = np.exp(gr * pos[:, 2])
            s0 = np.sum((b * c - a * d) * f)
            s1 = np.sum((c * a + b * d) * f)
            s2 = np.sum((-b * c - a * d) / f)
            s3 = np.sum((c * a - b * d) / f)
            e += fa1 * 2.0 * (s0 * s2 + s1 * s3)
    e *= -np.pi / (box[0] * box[1])
    vol = box[0] * box[1] * box[2]
    return prefactor * e + prefactor * 2.0 * np.pi / vol * np.sum(dip[:, 2]) ** 2


def dlc_force_correction(box, gap_size, pos, dip, prefactor, far_cut):
    """DLC force and torque corrections for a metallic base solver
    (DipolarLayerCorrection::add_force_corrections, dlc.cpp:304-354, with
    dipolar_force_corrections :111-245 after Brodka): per 2D wave vector the
    particle terms S_j(+-) and their position gradients against the sums S,
    scaled by pi / (L_x L_y) fa1 (g_x, g_y, g); torques mu x (sum), plus the
    shape torque mu x (0, 0, -4 pi / V M_z); all times the prefactor.
    Returns (forces, torques) for all particles (zero for non-magnetic)."""
    box = np.asarray(box, dtype=np.float64)
    pos = np.asarray(pos, dtype=np.float64)
    dip = np.asarray(dip, dtype=np.float64)
    n = len(pos)
    pos = pos - np.floor(pos / box) * box
    mag = np.linalg.norm(dip, axis=1) != 0.0
    kc = int(np.round(far_cut))
    fx, fy = 2.0 * np.pi / box[0], 2.0 * np.pi / box[1]
    fs = np.zeros((n, 3))
    ts = np.zeros((n, 3))
    for ix in range(-kc, kc + 1):
        for iy in range(-kc, kc + 1):
            if ix == 0 and iy == 0:
                continue
            gx, gy = ix * fx, iy * fy
            gr = np.sqrt(gx * gx + gy * gy)
            fa1 = 1.0 / (gr * (np.exp(gr * box[2]) - 1.0))
            a = gx * dip[:, 0] + gy * dip[:, 1]
            b = gr * dip[:, 2]
            er = gx * pos[:, 0] + gy * pos[:, 1]
            c, d = np.cos(er), np.sin(er)
            f = np.exp(gr * pos[:, 2])
            rp = np.where(mag, (b * c - a * d) * f, 0.0)
            ip = np.where(mag, (c * a + b * d) * f, 0.0)
            rm = np.where(mag, (-b * c - a * d) / f, 0.0)
            im = np.where(mag, (c * a - b * d) / f, 0.0)
            S = (rp.sum(), ip.sum(), rm.sum(), im.sum())
            for (xp, yp, xm, ym), acc in (((rp, ip, rm, im), fs),
                                          ((c * f, d * f, c / f, d / f), ts)):
                s1 = -(-xp * S[3] + yp * S[2])
                s2 = xm * S[1] - ym * S[0]
                s3 = -(-xm * S[1] + ym * S[0])
                s4 = xp * S[3] - yp * S[2]
                s1z = xp * S[2] + yp * S[3]
                s2z = -(xm * S[0] + ym * S[1])
                ss = np.where(mag, s1 + s2 + s3 + s4, 0.0)
                sz = np.where(mag, 2.0 * s1z + 2.0 * s2z, 0.0)
                acc[:, 0] += fa1 * gx * ss
                acc[:, 1] += fa1 * gy * ss
                acc[:, 2] += fa1 * gr * sz
    ts = np.cross(dip, ts)
    piarea = np.pi / (box[0] * box[1])
    fs *= piarea
    ts *= piarea
    vol = box[0] * box[1] * box[2]
    mz = np.sum(dip[mag, 2])
    shape = np.array([0.0, 0.0, -4.0 * np.pi / vol * mz])
    ts += np.where(mag[:, None], np.cross(dip, shape), 0.0)
    return prefactor * fs, prefactor * ts
