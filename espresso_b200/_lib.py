"""ctypes binding of libp3mx.so (the C ABI declared in include/p3mx.h).

The library is built in-tree for sm_100a (espresso_b200/build.py).  If it is
missing this module raises: there is no CPU fallback for the product path.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libp3mx.so")

P3MX_DEVICE_PTRS = 1
P3MX_FORCES = 2
P3MX_ENERGY = 4
P3MX_VIRIAL = 8
P3MX_OVERWRITE = 16
P3MX_MIXED_OBSERVABLES = 32

STATUS = {0: "OK", 1: "EDOMAIN", 2: "ERUNTIME", 3: "ECUDA", 4: "ENOMEM", 5: "EHANDLE"}


class Params(ctypes.Structure):
    _fields_ = [("prefactor", ctypes.c_double), ("accuracy", ctypes.c_double),
                ("mesh", ctypes.c_int * 3), ("cao", ctypes.c_int),
                ("r_cut", ctypes.c_double), ("alpha", ctypes.c_double),
                ("epsilon", ctypes.c_double), ("mesh_off", ctypes.c_double * 3),
                ("tune", ctypes.c_int), ("timings", ctypes.c_int),
                ("verbose", ctypes.c_int), ("single_precision", ctypes.c_int),
                ("check_neutrality", ctypes.c_int),
                ("charge_neutrality_tolerance", ctypes.c_double)]


class SystemDesc(ctypes.Structure):
    _fields_ = [("box", ctypes.c_double * 3), ("skin", ctypes.c_double),
                ("periodic", ctypes.c_int * 3)]


class Tuned(ctypes.Structure):
    _fields_ = [("mesh", ctypes.c_int * 3), ("cao", ctypes.c_int),
                ("r_cut", ctypes.c_double), ("alpha", ctypes.c_double),
                ("r_cut_iL", ctypes.c_double), ("alpha_L", ctypes.c_double),
                ("accuracy", ctypes.c_double), ("epsilon", ctypes.c_double),
                ("mesh_off", ctypes.c_double * 3), ("a", ctypes.c_double * 3),
                ("is_tuned", ctypes.c_int), ("single_precision", ctypes.c_int),
                ("rs_error", ctypes.c_double), ("ks_error", ctypes.c_double)]


class PairParams(ctypes.Structure):
    _fields_ = [("lj_eps", ctypes.c_double), ("lj_sig", ctypes.c_double),
                ("lj_cut", ctypes.c_double), ("lj_shift", ctypes.c_double),
                ("lj_offset", ctypes.c_double), ("lj_min", ctypes.c_double),
                ("wca_eps", ctypes.c_double), ("wca_sig", ctypes.c_double)]


P3MX_BOND_FENE = 1
P3MX_BOND_HARMONIC = 2


class BondParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("k", ctypes.c_double), ("r0", ctypes.c_double),
                ("r_max", ctypes.c_double)]


class ElcParams(ctypes.Structure):
    _fields_ = [("maxPWerror", ctypes.c_double), ("gap_size", ctypes.c_double),
                ("far_cut", ctypes.c_double), ("neutralize", ctypes.c_int),
                ("delta_mid_top", ctypes.c_double), ("delta_mid_bot", ctypes.c_double),
                ("const_pot", ctypes.c_int), ("pot_diff", ctypes.c_double)]


class BatchDesc(ctypes.Structure):
    _fields_ = [("n_rep", ctypes.c_int), ("box", ctypes.POINTER(ctypes.c_double)),
                ("prefactor", ctypes.POINTER(ctypes.c_double)),
                ("offset", ctypes.POINTER(ctypes.c_longlong)),
                ("accuracy", ctypes.c_double), ("skin", ctypes.c_double),
                ("single_precision", ctypes.c_int), ("mesh_min", ctypes.c_int),
                ("mesh_max", ctypes.c_int), ("cao_min", ctypes.c_int),
                ("cao_max", ctypes.c_int)]


class Dp3mParams(ctypes.Structure):
    _fields_ = [("prefactor", ctypes.c_double), ("accuracy", ctypes.c_double),
                ("mesh", ctypes.c_int * 3), ("cao", ctypes.c_int),
                ("r_cut", ctypes.c_double), ("alpha", ctypes.c_double),
                ("epsilon", ctypes.c_double), ("mesh_off", ctypes.c_double * 3),
                ("tune", ctypes.c_int), ("timings", ctypes.c_int),
                ("verbose", ctypes.c_int), ("single_precision", ctypes.c_int)]


# every symbol of include/p3mx.h, with its ctypes signature
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_sz = ctypes.c_size_t
SIGNATURES = {
    "p3mx_version": (ctypes.c_char_p, []),
    "p3mx_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.POINTER(_vp)]),
    "p3mx_destroy": (None, [_vp]),
    "p3mx_last_error": (ctypes.c_char_p, [_vp]),
    "p3mx_set_system": (ctypes.c_int, [_vp, ctypes.POINTER(SystemDesc)]),
    "p3mx_activate": (ctypes.c_int, [_vp, _sz, _vp, _vp, ctypes.c_uint]),
    "p3mx_get_tuned": (ctypes.c_int, [_vp, ctypes.POINTER(Tuned)]),
    "p3mx_long_range": (ctypes.c_int, [_vp, _sz, _vp, _vp, _vp, _dp, _dp, ctypes.c_uint, _vp]),
    "p3mx_set_pair_params": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(PairParams)]),
    "p3mx_set_bonds": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(BondParams), _sz,
                                      ctypes.POINTER(ctypes.c_int)]),
    "p3mx_bond_observables": (ctypes.c_int, [_vp, _sz, _vp, _dp, _dp, ctypes.c_uint, _vp]),
    "p3mx_set_elc": (ctypes.c_int, [_vp, ctypes.POINTER(ElcParams)]),
    "p3mx_get_elc": (ctypes.c_int, [_vp, _dp, _dp, ctypes.POINTER(ctypes.c_int)]),
    "p3mx_batch_set_bonds": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(BondParams), _sz,
                                            ctypes.POINTER(ctypes.c_int)]),
    "p3mx_batch_profile": (ctypes.c_int, [_vp, ctypes.c_int, _dp,
                                          ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]),
    "p3mx_short_range": (ctypes.c_int, [_vp, _sz, _vp, _vp, _vp, _vp, _dp, _dp, ctypes.c_uint, _vp]),
    "p3mx_forces": (ctypes.c_int, [_vp, _sz, _vp, _vp, _vp, _vp, _dp, _dp, ctypes.c_uint, _vp]),
    "p3mx_cell_grid": (ctypes.c_int, [_vp, _ip, _dp]),
    "p3mx_cell_index": (ctypes.c_int, [_vp, _sz, _dp, _ip]),
    "p3mx_verlet_pairs": (ctypes.c_int, [_vp, _sz, _dp, _dp, _ip, _ip, _sz, ctypes.POINTER(_sz)]),
    "p3mx_copy_mesh": (ctypes.c_int, [_vp, _dp, _sz]),
    "p3mx_profile": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_char_p),
                                    ctypes.c_int, _ip]),
    "p3mx_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "p3mx_resort": (ctypes.c_int, [_vp]),
    "p3mx_exp_check": (ctypes.c_int, [_sz, _vp, _vp, _vp]),
    "p3mx_error_estimate": (ctypes.c_int, [_ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, _dp, ctypes.c_double,
                                           _dp, _dp]),
    "p3mx_error_estimate_noalloc": (ctypes.c_int, [_ip, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_double, _dp,
                                                   ctypes.c_double, _dp, _dp, _vp, ctypes.c_char_p,
                                                   _sz]),
    "p3mx_batch_create": (ctypes.c_int, [ctypes.POINTER(BatchDesc), _dp, _dp, _ip, ctypes.c_int,
                                         ctypes.POINTER(PairParams), ctypes.POINTER(_vp)]),
    "p3mx_batch_destroy": (None, [_vp]),
    "p3mx_batch_last_error": (ctypes.c_char_p, [_vp]),
    "p3mx_batch_get_tuned": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(Tuned)]),
    "p3mx_batch_forces": (ctypes.c_int, [_vp, _dp]),
    "p3mx_batch_set_cao": (ctypes.c_int, [_vp, _ip]),
    "p3mx_batch_run": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_ulonglong]),
    "p3mx_batch_stream": (ctypes.c_void_p, [_vp]),
    "p3mx_batch_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    "p3mx_batch_get": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
    "p3mx_dp3m_create": (ctypes.c_int, [ctypes.POINTER(Dp3mParams), ctypes.POINTER(_vp)]),
    "p3mx_dp3m_destroy": (None, [_vp]),
    "p3mx_dp3m_last_error": (ctypes.c_char_p, [_vp]),
    "p3mx_dp3m_set_system": (ctypes.c_int, [_vp, ctypes.POINTER(SystemDesc)]),
    "p3mx_dp3m_activate": (ctypes.c_int, [_vp, _sz, _vp, _vp, ctypes.c_uint]),
    "p3mx_dp3m_get_tuned": (ctypes.c_int, [_vp, ctypes.POINTER(Tuned)]),
    "p3mx_dp3m_compute": (ctypes.c_int, [_vp, _sz, _vp, _vp, _vp, _vp, _dp, ctypes.c_uint, _vp]),
    "p3mx_dp3m_profile": (ctypes.c_int, [_vp, _sz, _vp, _vp, ctypes.c_int, _dp,
                                         ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, _ip]),
    "p3mx_dp3m_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
}

_lib = None


def load(build_if_missing=True):
    """Load (building first if needed) libp3mx.so; raise if unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH) and build_if_missing:
        from . import build
        build.build()
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libp3mx.so not found at {LIB_PATH}: build it with "
                           "`python -m espresso_b200.build` (no CPU fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class P3MXError(RuntimeError):
    pass


def check(rc, handle=None, fn_err=None):
    if rc == 0:
        return
    lib = load()
    msg = ""
    if handle is not None:
        msg = (fn_err or lib.p3mx_last_error)(handle)
        msg = msg.decode() if msg else ""
    if rc == 1:
        raise ValueError(msg)
    raise P3MXError(f"{STATUS.get(rc, rc)}: {msg}")


def dptr(a):
    """Host numpy array or torch CUDA tensor -> c_void_p."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    return a.ctypes.data_as(ctypes.c_void_p)


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)
