"""P3M electrostatics actors, a drop-in mirror of ``espressomd.electrostatics``.

``P3M`` and ``P3MGPU`` take the keyword arguments of the reference actors
(src/python/espressomd/electrostatics.py:129-284) with the same defaults,
validation and error messages; the computation runs in libp3mx.so on the GPU
(``single_precision=True`` selects the FP32-mixed mesh/FFT path,
``False`` the plain FP64 path).
"""
import ctypes

import numpy as np

from . import _lib

_METALLIC = 0.0


class _P3MBase:
    _defaults = {"cao": -1, "r_cut": -1., "alpha": -1., "mesh": [-1, -1, -1],
                 "epsilon": 0., "mesh_off": [-1., -1., -1.], "prefactor": 0.,
                 "check_neutrality": True, "check_complex_residuals": True,
                 "tune": True, "timings": 10, "verbose": True,
                 "charge_neutrality_tolerance": 2e-12}
    _single_precision_default = False

    def __init__(self, **kwargs):
        for key in ("prefactor", "accuracy"):
            if key not in kwargs:
                raise ValueError(f"At least the following keys have to be given as keyword "
                                 f"arguments: ['accuracy', 'prefactor'], got {sorted(kwargs)}")
        params = dict(self._defaults)
        params["single_precision"] = self._single_precision_default
        params.update(kwargs)
        self._validate(params)
        self._params = params
        self._handle = None
        self._create()

    # --- validation (electrostatics.py:150-184) ---------------------------
    @staticmethod
    def _validate(p):
        mesh = p["mesh"]
        if isinstance(mesh, (int, np.integer)):
            mesh = 3 * [int(mesh)]
        mesh = list(mesh)
        if len(mesh) != 3 or not all(isinstance(m, (int, np.integer)) for m in mesh):
            raise ValueError("Parameter 'mesh' has to be an integer or integer list of length 3")
        if any(m % 2 != 0 and m != -1 for m in mesh):
            raise ValueError("P3M requires an even number of mesh points in all directions")
        p["mesh"] = [int(m) for m in mesh]
        if p["epsilon"] == "metallic":
            p["epsilon"] = _METALLIC
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
        if not p.get("check_neutrality", True):
            p["charge_neutrality_tolerance"] = -1.0

    def _create(self):
        lib = _lib.load()
        p = self._params
        c = _lib.Params()
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
        c.check_neutrality = 1 if p["check_neutrality"] else 0
        c.charge_neutrality_tolerance = float(p["charge_neutrality_tolerance"])
        h = ctypes.c_void_p()
        rc = lib.p3mx_create(ctypes.byref(c), ctypes.byref(h))
        if rc != 0:
            msg = lib.p3mx_last_error(h).decode() if h.value else ""
            if h.value:
                lib.p3mx_destroy(h)
            if rc == 1:
                raise ValueError(msg)
            raise _lib.P3MXError(msg)
        self._handle = h

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value and _lib._lib is not None:
            _lib._lib.p3mx_destroy(h)
            self._handle = None

    # --- read-only parameter view (CoulombP3M.hpp:67-99) ------------------
    def _tuned(self):
        t = _lib.Tuned()
        _lib.check(_lib.load().p3mx_get_tuned(self._handle, ctypes.byref(t)), self._handle)
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

    # --- checkpointing ----------------------------------------------------
    # As the reference's script-interface checkpoints, a pickled actor keeps
    # its parameters with the tuned values (mesh, cao, r_cut, alpha,
    # mesh_off, achieved accuracy); the restored actor does not tune again.
    def __reduce__(self):
        p = dict(self._params)
        if self._handle is not None and self._handle.value:
            t = self._tuned()
            if t.is_tuned:
                p.update(mesh=[int(m) for m in t.mesh], cao=int(t.cao), r_cut=float(t.r_cut),
                         alpha=float(t.alpha), mesh_off=[float(x) for x in t.mesh_off],
                         accuracy=float(t.accuracy), tune=False)
        return (_restore_actor, (type(self), p))

    # --- engine-facing calls ---------------------------------------------
    def _set_system(self, box_l, skin, periodicity):
        s = _lib.SystemDesc()
        for d in range(3):
            s.box[d] = float(box_l[d])
            s.periodic[d] = 1 if periodicity[d] else 0
        s.skin = float(skin)
        _lib.check(_lib.load().p3mx_set_system(self._handle, ctypes.byref(s)), self._handle)

    def _activate(self, pos, q):
        pos = _lib.as_f64(pos)
        q = _lib.as_f64(q)
        rc = _lib.load().p3mx_activate(self._handle, len(q), _lib.dptr(pos), _lib.dptr(q), 0)
        _lib.check(rc, self._handle)

    def _detach_layer_correction(self):
        # the actor used on its own again: no ELC on its handle
        _lib.check(_lib.load().p3mx_set_elc(self._handle, None), self._handle)


class P3M(_P3MBase):
    """P3M electrostatics solver (plain FP64 path unless single_precision)."""
    _so_name = "Coulomb::CoulombP3M"
    _single_precision_default = False


class P3MGPU(_P3MBase):
    """P3M electrostatics solver with the FP32-mixed GPU path by default."""
    _so_name = "Coulomb::CoulombP3MGPU"
    _single_precision_default = True


def _restore_actor(cls, params):
    return cls(**params)


def _real(x):
    return isinstance(x, (float, int, np.floating, np.integer)) and not isinstance(x, bool)


class ELC:
    """Electrostatic layer correction for slab systems (2D-periodic, with an
    empty gap along z), a mirror of ``espressomd.electrostatics.ELC``
    (src/python/espressomd/electrostatics.py:288-365): same keyword
    arguments, defaults and checks.  The base ``actor`` (P3M or P3MGPU)
    computes the 3D-periodic solution and the correction runs in FP64 CUDA
    kernels of libp3mx.so; with dielectric contrasts (``delta_mid_top`` /
    ``delta_mid_bot`` != 0, optionally ``const_pot``) the mesh also carries
    the image charges (in FP64 for both actors) and the short-range loop the
    image-layer corrections.
    """
    _so_name = "Coulomb::ElectrostaticLayerCorrection"
    _defaults = {"far_cut": -1., "delta_mid_top": 0., "delta_mid_bot": 0.,
                 "const_pot": False, "pot_diff": 0., "neutralize": True,
                 "check_neutrality": True}
    _required = ("actor", "gap_size", "maxPWerror")

    def __init__(self, **kwargs):
        if any(k not in kwargs for k in self._required):
            raise ValueError(f"At least the following keys have to be given as keyword "
                             f"arguments: {sorted(self._required)}, got {sorted(kwargs)}")
        p = dict(self._defaults)
        p.update(kwargs)
        for key in ("maxPWerror", "gap_size", "far_cut"):
            if not _real(p[key]):
                raise TypeError(f"{key} has to be a float")
        if not isinstance(p["neutralize"], (bool, np.bool_)):
            raise TypeError("neutralize has to be a bool")
        if not isinstance(p["actor"], _P3MBase):
            raise TypeError("ELC requires a P3M or P3MGPU actor")
        self._params = p
        self._attach()

    @property
    def actor(self):
        return self._params["actor"]

    @property
    def _handle(self):
        return self.actor._handle

    def _attach(self):
        p = self._params
        c = _lib.ElcParams()
        c.maxPWerror = float(p["maxPWerror"])
        c.gap_size = float(p["gap_size"])
        c.far_cut = float(p["far_cut"])
        c.neutralize = 1 if p["neutralize"] else 0
        c.delta_mid_top = float(p["delta_mid_top"])
        c.delta_mid_bot = float(p["delta_mid_bot"])
        c.const_pot = 1 if p["const_pot"] else 0
        c.pot_diff = float(p["pot_diff"])
        _lib.check(_lib.load().p3mx_set_elc(self._handle, ctypes.byref(c)), self._handle)
        # adapt_epsilon_elc: the base actor is metallic from now on
        self.actor._params["epsilon"] = _METALLIC

    def get_params(self):
        out = dict(self._params)
        fc = ctypes.c_double()
        if _lib.load().p3mx_get_elc(self._handle, ctypes.byref(fc), None, None) == 0:
            out["far_cut"] = fc.value
        return out

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        params = self.__dict__.get("_params", {})
        if name == "far_cut":
            return self.get_params()["far_cut"]
        if name in params:
            return params[name]
        raise AttributeError(name)

    def __reduce__(self):
        return (_restore_actor, (type(self), dict(self._params)))

    # --- engine-facing calls: the base actor's, then ELC's activation
    # (ElectrostaticLayerCorrection::on_activation: checks, box_h, far_cut)
    def _set_system(self, box_l, skin, periodicity):
        self.actor._set_system(box_l, skin, periodicity)

    def _activate(self, pos, q):
        self.actor._activate(pos, q)
        self._attach()
