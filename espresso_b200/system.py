"""Minimal host-side system mirroring the slice of ``espressomd.System`` that
the P3M + short-range force path needs: particles (pos, q, type, v, f), box,
periodicity, Verlet skin, LJ/WCA parameters, FENE / harmonic bonds, the
electrostatics and magnetostatics containers (point dipoles in ``dip``,
torques in ``torque_lab``),
``integrator.run`` and ``analysis.energy/pressure/pressure_tensor``.

Every force, energy and virial comes from libp3mx.so through the C ABI
(p3mx_forces / p3mx_short_range); this module only keeps host arrays and
mirrors the reference's observable bookkeeping (energy.cpp:39-111,
pressure.cpp:46-123).  The integrator here is a host-side velocity Verlet
for scripting convenience; the device-resident integrator lives in the
batched engine.
"""
import ctypes

import numpy as np

from . import _lib
from .electrostatics import ELC, P3M, _P3MBase
from .interactions import BondedInteractions
from .magnetostatics import Magnetostatics


class CellSystem:
    def __init__(self, system=None):
        self.skin = 0.4
        self.use_verlet_lists = True
        self._system = system

    def set_regular_decomposition(self, use_verlet_lists=True):
        self.use_verlet_lists = use_verlet_lists

    def resort(self):
        """Rebuild the cell and Verlet lists at the next force calculation
        (CellSystem.resort() of the reference, cell_system.py; the next
        step rebuilds as after CellStructure::set_resort_particles)."""
        s = self._system
        if s is None:
            return
        handles = [getattr(a, "_handle", None) for a in (s.electrostatics.solver, s._sr_handle)
                   if a is not None]
        lib = _lib.load()
        for h in handles:
            if h:
                _lib.check(lib.p3mx_resort(h), h)


class _PairIA:
    def __init__(self):
        self.lj = dict(epsilon=0.0, sigma=0.0, cutoff=0.0, shift=0.0, offset=0.0, min=0.0)
        self.wca = dict(epsilon=0.0, sigma=0.0)


class _LJHandle:
    def __init__(self, ia, owner):
        self._ia, self._owner = ia, owner

    def set_params(self, epsilon, sigma, cutoff, shift=0.0, offset=0.0, min=0.0):
        if epsilon < 0:
            raise ValueError("LJ parameter 'epsilon' has to be >= 0")
        if sigma < 0:
            raise ValueError("LJ parameter 'sigma' has to be >= 0")
        if cutoff < 0:
            raise ValueError("LJ parameter 'cutoff' has to be >= 0")
        if shift == "auto":
            # shift so that the energy vanishes at the cutoff (lj.py semantics)
            shift = -((sigma / cutoff) ** 12 - (sigma / cutoff) ** 6) if cutoff > 0 else 0.0
        self._ia.lj = dict(epsilon=float(epsilon), sigma=float(sigma), cutoff=float(cutoff),
                           shift=float(shift), offset=float(offset), min=float(max(min, 0.0)))
        self._owner._changed()

    def get_params(self):
        return dict(self._ia.lj)


class _WCAHandle:
    def __init__(self, ia, owner):
        self._ia, self._owner = ia, owner

    def set_params(self, epsilon, sigma):
        if epsilon < 0:
            raise ValueError("WCA parameter 'epsilon' has to be >= 0")
        if sigma < 0:
            raise ValueError("WCA parameter 'sigma' has to be >= 0")
        self._ia.wca = dict(epsilon=float(epsilon), sigma=float(sigma))
        self._owner._changed()

    @property
    def cutoff(self):
        return self._ia.wca["sigma"] * 2 ** (1 / 6) if self._ia.wca["sigma"] else 0.0

    def get_params(self):
        return dict(self._ia.wca, cutoff=self.cutoff)


class _PairView:
    def __init__(self, ia, owner):
        self.lennard_jones = _LJHandle(ia, owner)
        self.wca = _WCAHandle(ia, owner)


class NonBondedInteractions:
    def __init__(self, system):
        self._system = system
        self._table = {}

    def __getitem__(self, key):
        a, b = sorted(key)
        ia = self._table.setdefault((a, b), _PairIA())
        return _PairView(ia, self)

    def _changed(self):
        self._system._pairs_dirty = True

    def ntypes(self, types):
        nt = 1 + max([max(k) for k in self._table] + [int(types.max()) if len(types) else 0])
        return nt

    def c_table(self, ntypes):
        tab = (_lib.PairParams * (ntypes * ntypes))()
        for (a, b), ia in self._table.items():
            for (x, y) in ((a, b), (b, a)):
                e = tab[x * ntypes + y]
                e.lj_eps, e.lj_sig = ia.lj["epsilon"], ia.lj["sigma"]
                e.lj_cut, e.lj_shift = ia.lj["cutoff"], ia.lj["shift"]
                e.lj_offset, e.lj_min = ia.lj["offset"], ia.lj["min"]
                e.wca_eps, e.wca_sig = ia.wca["epsilon"], ia.wca["sigma"]
        return tab

    def active(self):
        return any((ia.lj["epsilon"] > 0 and ia.lj["cutoff"] > 0) or
                   (ia.wca["epsilon"] > 0 and ia.wca["sigma"] > 0)
                   for ia in self._table.values())


class ParticleHandle:
    def __init__(self, plist, idx):
        self._pl, self._idx = plist, idx

    def __getattr__(self, name):
        if name in ("pos", "f", "v", "q", "type", "mass", "dip"):
            arr = getattr(self._pl, "_" + name)
            return np.copy(arr[self._idx])
        if name == "torque_lab":
            return np.copy(self._pl._torque[self._idx])
        if name == "dipm":
            return np.linalg.norm(self._pl._dip[self._idx], axis=-1)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in ("pos", "f", "v", "q", "type", "mass", "dip"):
            getattr(self._pl, "_" + name)[self._idx] = value
            self._pl._system._touch(name)
        else:
            object.__setattr__(self, name, value)

    @property
    def id(self):
        return int(np.atleast_1d(self._idx)[0]) if np.ndim(self._idx) == 0 else None

    def _index(self):
        if isinstance(self._idx, slice) or np.ndim(self._idx) != 0:
            raise ValueError("bonds belong to single particles")
        return int(self._idx)

    def add_bond(self, bond):
        """bond = (bond object, partner particle or id), as in espressomd."""
        obj, partner = bond
        j = partner._index() if isinstance(partner, ParticleHandle) else int(partner)
        self._pl._system.bonded_inter._id(obj)
        i = self._index()
        if not 0 <= j < len(self._pl):
            raise ValueError("bond partner %d does not exist" % j)
        self._pl._bonds.append((obj, i, j))
        self._pl._system._bonds_changed()

    @property
    def bonds(self):
        i = self._index()
        return tuple((obj, j) for obj, a, j in self._pl._bonds if a == i)

    @bonds.setter
    def bonds(self, value):
        i = self._index()
        self._pl._bonds = [b for b in self._pl._bonds if b[1] != i]
        self._pl._system._bonds_changed()
        for bond in value:
            self.add_bond(bond)


class ParticleList:
    def __init__(self, system):
        self._system = system
        self.clear()

    def clear(self):
        self._pos = np.zeros((0, 3))
        self._v = np.zeros((0, 3))
        self._f = np.zeros((0, 3))
        self._q = np.zeros(0)
        self._type = np.zeros(0, dtype=np.int32)
        self._mass = np.zeros(0)
        self._dip = np.zeros((0, 3))
        self._torque = np.zeros((0, 3))
        self._bonds = []  # (bond object, owner index, partner index)
        self._system._touch("all")
        if hasattr(self._system, "_bond_version"):
            self._system._bonds_changed()

    def add(self, pos, q=None, type=None, v=None, mass=None, dip=None):
        pos = np.asarray(pos, dtype=float)
        single = pos.ndim == 1
        pos = np.atleast_2d(pos)
        n = len(pos)

        def col(val, default, shape, dtype=float):
            if val is None:
                return np.full(shape, default, dtype=dtype)
            return np.broadcast_to(np.asarray(val, dtype=dtype), shape).copy()

        i0 = len(self._q)
        self._pos = np.vstack([self._pos, pos])
        self._v = np.vstack([self._v, col(v, 0.0, (n, 3))])
        self._f = np.vstack([self._f, np.zeros((n, 3))])
        self._q = np.concatenate([self._q, col(q, 0.0, (n,))])
        self._type = np.concatenate([self._type, col(type, 0, (n,), np.int32)])
        self._mass = np.concatenate([self._mass, col(mass, 1.0, (n,))])
        self._dip = np.vstack([self._dip, col(dip, 0.0, (n, 3))])
        self._torque = np.vstack([self._torque, np.zeros((n, 3))])
        self._system._touch("all")
        return ParticleHandle(self, i0 if single else slice(i0, i0 + n))

    def all(self):
        return ParticleHandle(self, slice(0, len(self._q)))

    def by_id(self, i):
        return ParticleHandle(self, int(i))

    def __len__(self):
        return len(self._q)

    def __iter__(self):
        for i in range(len(self._q)):
            yield ParticleHandle(self, i)


class Electrostatics:
    def __init__(self, system):
        self._system = system
        self._solver = None

    @property
    def solver(self):
        return self._solver

    @solver.setter
    def solver(self, actor):
        if actor is None:
            self.clear()
            return
        if not isinstance(actor, (_P3MBase, ELC)):
            raise TypeError("only P3M / P3MGPU / ELC actors are supported")
        s = self._system
        if s.time_step is None:
            raise RuntimeError("time_step not set")
        if isinstance(actor, _P3MBase):
            actor._detach_layer_correction()
        actor._set_system(s.box_l, s.cell_system.skin, s.periodicity)
        actor._activate(s.part._pos, s.part._q)  # raises and leaves no solver on failure
        self._solver = actor
        s._pairs_dirty = True

    def clear(self):
        self._solver = None
        self._system._pairs_dirty = True


class Thermostat:
    """Langevin thermostat of the velocity-Verlet integrator, mirroring
    ``espressomd.thermostat.Thermostat.set_langevin`` (thermostats/
    langevin_inline.hpp:40-59): at every force calculation each particle
    gets the friction -gamma v and a noise force of uniform components
    sqrt(24 kT gamma / dt) (U(0, 1) - 1/2), drawn from a counter-based
    Philox stream keyed by the seed (deterministic for a given seed)."""

    def __init__(self):
        self.kT = None
        self.gamma = None
        self.seed = None
        self._rng = None

    def set_langevin(self, kT, gamma, seed):
        if kT < 0 or gamma < 0:
            raise ValueError("kT and gamma must be >= 0")
        self.kT, self.gamma, self.seed = float(kT), float(gamma), int(seed)
        self._rng = np.random.Generator(np.random.Philox(key=self.seed))

    def turn_off(self):
        self.kT = self.gamma = self.seed = None
        self._rng = None

    def _forces(self, v, dt):
        if self._rng is None or not self.gamma:
            return 0.0
        noise = np.sqrt(24.0 * self.kT * self.gamma / dt)
        return -self.gamma * v + noise * (self._rng.random(v.shape) - 0.5)


class Integrator:
    def __init__(self, system):
        self._system = system

    def run(self, steps=1, recalc_forces=False):
        """Velocity Verlet (integrators/velocity_verlet_inline.hpp:34-58)
        with the Langevin forces of ``system.thermostat`` added to the
        conservative forces from libp3mx.so at every step."""
        s = self._system
        if s.time_step is None:
            raise RuntimeError("time_step not set")
        dt = s.time_step
        s._calc_forces()
        s.part._f = s.part._f + s.thermostat._forces(s.part._v, dt)
        for _ in range(int(steps)):
            m = s.part._mass[:, None]
            s.part._v += 0.5 * dt * s.part._f / m
            s.part._pos += dt * s.part._v
            s._calc_forces()
            s.part._f = s.part._f + s.thermostat._forces(s.part._v, dt)
            s.part._v += 0.5 * dt * s.part._f / m


class Analysis:
    def __init__(self, system):
        self._system = system

    def energy(self):
        s = self._system
        e3, _ = s._calc_observables(energy=True)
        kin = 0.5 * float((s.part._mass[:, None] * s.part._v ** 2).sum())
        eb, _ = s._bond_observables()
        out = {"kinetic": kin, "coulomb": e3[0] + e3[1], "non_bonded": e3[2],
               "bonded": eb, "dipolar": s._e_dipolar}
        out["total"] = (kin + out["coulomb"] + out["non_bonded"] + out["bonded"] +
                        out["dipolar"])
        return out

    def pressure_tensor(self):
        s = self._system
        _, v27 = s._calc_observables(virial=True)
        V = float(np.prod(s.box_l))
        kin = np.einsum("i,ij,ik->jk", s.part._mass, s.part._v, s.part._v)
        _, vb = s._bond_observables()
        out = {"kinetic": kin / V, "coulomb": (v27[0] + v27[1]) / V,
               "non_bonded": v27[2] / V, "bonded": vb / V}
        out["total"] = out["kinetic"] + out["coulomb"] + out["non_bonded"] + out["bonded"]
        return out

    def pressure(self):
        return {k: float(np.trace(v)) / 3.0 for k, v in self.pressure_tensor().items()}


class System:
    """Host-side system holding particles; forces come from libp3mx.so."""

    def __init__(self, box_l):
        self._box_l = np.array(np.broadcast_to(box_l, (3,)), dtype=float)
        self.periodicity = (True, True, True)
        self.time_step = None
        self.cell_system = CellSystem(self)
        self.thermostat = Thermostat()
        self._sr_handle = None
        self._pairs_dirty = True
        self._bond_version = 0
        self.part = ParticleList(self)
        self.bonded_inter = BondedInteractions(self)
        self.non_bonded_inter = NonBondedInteractions(self)
        self.electrostatics = Electrostatics(self)
        self.magnetostatics = Magnetostatics(self)
        self._e_dipolar = 0.0
        self.integrator = Integrator(self)
        self.analysis = Analysis(self)

    @property
    def box_l(self):
        return self._box_l.copy()

    @box_l.setter
    def box_l(self, value):
        self._box_l = np.array(np.broadcast_to(value, (3,)), dtype=float)
        if self.electrostatics.solver is not None:
            self.electrostatics.solver._set_system(self._box_l, self.cell_system.skin,
                                                   self.periodicity)
        if self.magnetostatics.solver is not None:
            self.magnetostatics.solver._set_system(self._box_l, self.cell_system.skin,
                                                   self.periodicity)
        self._sr_handle = None

    def volume(self):
        return float(np.prod(self._box_l))

    # checkpointing: particles, interactions and the solver's (tuned)
    # parameters; the restored system activates its solver anew
    def __getstate__(self):
        st = dict(self.__dict__)
        st["_sr_handle"] = None
        st["_restore_solver"] = self.electrostatics._solver
        st["_restore_dipolar"] = self.magnetostatics._solver
        return st

    def __setstate__(self, st):
        solver = st.pop("_restore_solver")
        dipolar = st.pop("_restore_dipolar", None)
        self.__dict__.update(st)
        self.electrostatics._solver = None
        self.magnetostatics._solver = None
        if solver is not None:
            self.electrostatics.solver = solver
        if dipolar is not None:
            self.magnetostatics.solver = dipolar

    def _touch(self, what):
        pass

    def _bonds_changed(self):
        self._bond_version += 1

    def _sync_bonds(self, actor):
        """Send the bond list to the actor's handle when it changed since the
        last call on that actor (p3mx_set_bonds)."""
        if getattr(actor, "_bonds_of", None) is self and actor._bond_version == self._bond_version:
            return
        handle = actor._handle
        bonds = self.part._bonds
        kinds = self.bonded_inter
        types = (_lib.BondParams * max(1, len(kinds)))()
        for t in range(len(kinds)):
            types[t] = kinds[t].c_params()
        trip = np.array([(kinds._id(o), i, j) for o, i, j in bonds], dtype=np.int32).reshape(-1)
        rc = _lib.load().p3mx_set_bonds(
            handle, len(kinds), types, len(bonds),
            trip.ctypes.data_as(ctypes.POINTER(ctypes.c_int)) if len(bonds) else None)
        _lib.check(rc, handle)
        actor._bonds_of, actor._bond_version = self, self._bond_version

    def _force_actor(self):
        """Actor whose handle takes the force calls: the Coulomb solver, else
        the short-range one when pair or bonded interactions exist."""
        if self.electrostatics.solver is not None:
            return self.electrostatics.solver
        if (self.non_bonded_inter.active() or self.part._bonds) and len(self.part) > 0:
            return self._short_range_handle()
        return None

    def _bond_observables(self):
        """Bonded energy and virial tensor (sum of F (x) d)."""
        if not self.part._bonds:
            return 0.0, np.zeros((3, 3))
        act = self._force_actor()
        self._sync_bonds(act)
        h = act._handle
        pos = _lib.as_f64(self.part._pos)
        e = np.zeros(1)
        v = np.zeros(9)
        rc = _lib.load().p3mx_bond_observables(h, len(self.part), _lib.dptr(pos),
                                               e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               0, None)
        _lib.check(rc, h)
        return float(e[0]), v.reshape(3, 3)

    # -- force engine plumbing --------------------------------------------
    def _short_range_handle(self):
        """Handle used when no Coulomb solver is active (LJ/WCA only)."""
        if self._sr_handle is None:
            act = P3M(prefactor=1.0, accuracy=1.0, mesh=8, cao=1, r_cut=1e-6, alpha=1.0,
                      tune=False, check_neutrality=False)
            act._set_system(self._box_l, self.cell_system.skin, self.periodicity)
            act._activate(self.part._pos, np.zeros(len(self.part)))
            self._sr_handle = act
        return self._sr_handle

    def _sync_pairs(self, handle, types):
        nt = self.non_bonded_inter.ntypes(types)
        tab = self.non_bonded_inter.c_table(nt)
        _lib.check(_lib.load().p3mx_set_pair_params(handle, nt, tab), handle)

    def _run(self, energy=False, virial=False, forces=True):
        lib = _lib.load()
        n = len(self.part)
        pos = _lib.as_f64(self.part._pos)
        q = _lib.as_f64(self.part._q)
        t = np.ascontiguousarray(self.part._type, dtype=np.int32)
        f = np.zeros((n, 3))
        e3 = np.zeros(3)
        v27 = np.zeros(27)
        flags = _lib.P3MX_OVERWRITE | (_lib.P3MX_FORCES if forces else 0)
        flags |= (_lib.P3MX_ENERGY if energy else 0) | (_lib.P3MX_VIRIAL if virial else 0)
        solver = self.electrostatics.solver
        if solver is not None:
            h = solver._handle
            self._sync_pairs(h, t)
            self._sync_bonds(solver)
            rc = lib.p3mx_forces(h, n, _lib.dptr(pos), _lib.dptr(q), _lib.dptr(t), _lib.dptr(f),
                                 e3.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                 v27.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), flags, None)
            _lib.check(rc, h)
        elif (self.non_bonded_inter.active() or self.part._bonds) and n > 0:
            act = self._short_range_handle()
            h = act._handle
            self._sync_pairs(h, t)
            self._sync_bonds(act)
            e2 = np.zeros(2)
            v18 = np.zeros(18)
            zero_q = np.zeros(n)
            rc = lib.p3mx_short_range(h, n, _lib.dptr(pos), _lib.dptr(zero_q), _lib.dptr(t),
                                      _lib.dptr(f),
                                      e2.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      v18.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      flags, None)
            _lib.check(rc, h)
            e3[2] = e2[1]
            v27[18:] = v18[9:]
        # dipolar P3M: forces added, torques stored, energy returned apart
        self._e_dipolar = 0.0
        mag = self.magnetostatics.solver
        if mag is not None and n > 0 and (forces or energy):
            fd, td, ed = mag._compute(self.part._pos, self.part._dip, forces=forces,
                                      energy=energy)
            if forces:
                f += fd
                self.part._torque = td
            if energy:
                self._e_dipolar = ed
        return f, e3, v27.reshape(3, 3, 3)

    def _calc_forces(self):
        f, _, _ = self._run()
        self.part._f = f

    def _calc_observables(self, energy=False, virial=False):
        _, e3, v27 = self._run(energy=energy, virial=virial, forces=False)
        return e3, v27
