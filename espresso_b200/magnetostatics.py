"""Dipolar P3M, a drop-in mirror of ``espressomd.magnetostatics.DipolarP3M``.

``DipolarP3M`` takes the keyword arguments of the reference actor
(src/python/espressomd/magnetostatics.py:82-160) with the same defaults,
validation and error messages; the computation runs in libp3mx.so on the GPU
(``single_precision=True`` selects the FP32 mesh/FFT path with FP32
real-space pair terms summed in FP64, ``False`` the FP64 path).  It is activated with
``system.magnetostatics.solver = DipolarP3M(...)``; particles carry their
moments in ``dip`` and receive ``torque_lab``.
"""
import ctypes

import numpy as np

from . import _lib


class DipolarP3M:
    """Dipolar P3M solver (magnetostatics/dp3m.cpp) on the GPU."""
    _so_name = "Dipoles::DipolarP3M"
    _required = ("accuracy",)

    @staticmethod
    def default_params():
        return {"cao": -1, "r_cut": -1, "alpha": -1, "accuracy": -1,
                "mesh": [-1, -1, -1], "epsilon": 0.0, "mesh_off": [0.5, 0.5, 0.5],
                "prefactor": 0., "single_precision": False, "tune": True,
                "timings": 10, "verbose": True}

    def __init__(self, **kwargs):
        # MagnetostaticInteraction.__init__ (magnetostatics.py:44-60)
        for key in self._required:
            if key not in kwargs:
                raise RuntimeError(f"Parameter '{key}' is missing")
        params = self.default_params()
        params.update(kwargs)
        self._validate(params)
        for key in params:
            if key not in self.default_params():
                raise RuntimeError(f"Parameter '{key}' is not a valid parameter")
        self._params = params
        self._handle = None
        self._create()

    # --- validation (magnetostatics.py:61-65, 116-143) --------------------
    @staticmethod
    def _validate(p):
        pf = p["prefactor"]
        if not isinstance(pf, (float, int, np.floating, np.integer)) or isinstance(pf, bool):
            raise ValueError("Parameter 'prefactor' should be a float")
        mesh = p["mesh"]
        if isinstance(mesh, (int, np.integer)) and not isinstance(mesh, bool):
            p["mesh"] = 3 * [int(mesh)]
        else:
            mesh = list(mesh) if hasattr(mesh, "__len__") else [mesh]
            if len(mesh) != 3 or not all(isinstance(m, (int, np.integer)) for m in mesh):
                raise ValueError("Parameter 'mesh' has to be an integer or integer list of "
                                 "length 3")
            p["mesh"] = [int(m) for m in mesh]
        if p["epsilon"] == "metallic":
            p["epsilon"] = 0.0
        if not isinstance(p["epsilon"], (float, int, np.floating, np.integer)):
            raise ValueError("Parameter 'epsilon' has to be a float or 'metallic'")
        p["epsilon"] = float(p["epsilon"])
        mo = np.asarray(p["mesh_off"], dtype=float)
        if mo.shape != (3,):
            raise ValueError("Parameter 'mesh_off' has to be a (3,) array_like of values "
                             "between 0.0 and 1.0")
        p["mesh_off"] = [float(x) for x in mo]
        if not isinstance(p["timings"], (int, np.integer)) or isinstance(p["timings"], bool):
            raise TypeError("Parameter 'timings' has to be an integer")
        if not isinstance(p["tune"], (bool, np.bool_)):
            raise TypeError("Parameter 'tune' has to be a boolean")

    def _create(self):
        lib = _lib.load()
        p = self._params
        c = _lib.Dp3mParams()
        c.prefactor = float(p["prefactor"])
        c.accuracy = float(p["accuracy"])
        for d in range(3):
            c.mesh[d] = int(p["mesh"][d])
            c.mesh_off[d] = float(p["mesh_off"][d])
        c.cao = int(p["cao"])
        c.r_cut = float(p["r_cut"])
        c.alpha = float(p["alpha"])
        c.epsilon = float(p["epsilon"])
        c.tune = 1 if p["tune"] else 0
        c.timings = int(p["timings"])
        c.verbose = 1 if p["verbose"] else 0
        c.single_precision = 1 if p["single_precision"] else 0
        h = ctypes.c_void_p()
        rc = lib.p3mx_dp3m_create(ctypes.byref(c), ctypes.byref(h))
        if rc != 0:
            msg = lib.p3mx_dp3m_last_error(h).decode() if h.value else ""
            if h.value:
                lib.p3mx_dp3m_destroy(h)
            if rc == 1:
                raise ValueError(msg)
            raise _lib.P3MXError(msg)
        self._handle = h

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.p3mx_dp3m_destroy(h)
            self._handle = None

    def _check(self, rc):
        _lib.check(rc, self._handle, _lib.load().p3mx_dp3m_last_error)

    # --- read-only parameter view (script_interface DipolarP3M.hpp:60-92)
    def _tuned(self):
        t = _lib.Tuned()
        self._check(_lib.load().p3mx_dp3m_get_tuned(self._handle, ctypes.byref(t)))
        return t

    def get_params(self):
        t = self._tuned()
        out = dict(self._params)
        out.update(mesh=list(t.mesh), cao=t.cao, r_cut=t.r_cut, alpha=t.alpha,
                   accuracy=t.accuracy, alpha_L=t.alpha_L, r_cut_iL=t.r_cut_iL,
                   mesh_off=list(t.mesh_off), a=list(t.a), is_tuned=bool(t.is_tuned))
        return out

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        if name in ("mesh", "cao", "r_cut", "alpha", "accuracy", "alpha_L", "r_cut_iL",
                    "mesh_off", "a", "is_tuned"):
            return self.get_params()[name]
        if name in self._params:
            return self._params[name]
        raise AttributeError(name)

    def get_magnetostatics_prefactor(self):
        return self._params["prefactor"]

    # checkpointing: the tuned parameters travel, the restored actor does
    # not tune again
    def __reduce__(self):
        p = dict(self._params)
        if self._handle is not None and self._handle.value:
            t = self._tuned()
            if t.is_tuned:
                p.update(mesh=[int(m) for m in t.mesh], cao=int(t.cao), r_cut=float(t.r_cut),
                         alpha=float(t.alpha), mesh_off=[float(x) for x in t.mesh_off],
                         accuracy=float(t.accuracy), tune=False)
        return (_restore, (type(self), p))

    # --- engine-facing calls ---------------------------------------------
    def _set_system(self, box_l, skin, periodicity):
        s = _lib.SystemDesc()
        for d in range(3):
            s.box[d] = float(box_l[d])
            s.periodic[d] = 1 if periodicity[d] else 0
        s.skin = float(skin)
        self._check(_lib.load().p3mx_dp3m_set_system(self._handle, ctypes.byref(s)))

    def _activate(self, pos, dip):
        pos = _lib.as_f64(pos)
        dip = _lib.as_f64(dip)
        self._check(_lib.load().p3mx_dp3m_activate(self._handle, len(pos), _lib.dptr(pos),
                                                   _lib.dptr(dip), 0))

    def _compute(self, pos, dip, forces=True, energy=False, overwrite=True):
        """Host arrays in, (forces, torques, energy) out; forces and torques
        are None when not requested, energy the total dipolar energy
        (k-space with its corrections plus real space) or None."""
        pos = _lib.as_f64(pos)
        dip = _lib.as_f64(dip)
        n = len(pos)
        f = np.zeros((n, 3)) if forces else None
        t = np.zeros((n, 3)) if forces else None
        e = np.zeros(2)
        flags = (_lib.P3MX_FORCES if forces else 0) | (_lib.P3MX_ENERGY if energy else 0)
        flags |= _lib.P3MX_OVERWRITE if overwrite else 0
        rc = _lib.load().p3mx_dp3m_compute(self._handle, n, _lib.dptr(pos), _lib.dptr(dip),
                                           _lib.dptr(f), _lib.dptr(t),
                                           e.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                           flags, None)
        self._check(rc)
        return f, t, (float(e[0] + e[1]) if energy else None)


def _restore(cls, params):
    return cls(**params)


class Magnetostatics:
    """``system.magnetostatics``: holds the active dipolar solver
    (Dipoles::Container, magnetostatics.py:25-29)."""

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
        if not isinstance(actor, DipolarP3M):
            raise TypeError("only the DipolarP3M actor is supported")
        s = self._system
        if s.time_step is None:
            raise RuntimeError("time_step not set")
        actor._set_system(s.box_l, s.cell_system.skin, s.periodicity)
        actor._activate(s.part._pos, s.part._dip)  # raises and leaves no solver on failure
        self._solver = actor

    def clear(self):
        self._solver = None
