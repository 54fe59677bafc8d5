"""ctypes binding of include/mlegs_b200.h (the library's C ABI).

This is the binding a Python host of the reference path would add; the
Fortran host binds the same symbols through ISO_C_BINDING.
The library is loaded from the package directory only: there is no CPU
fallback, and a missing or unloadable library raises immediately.
"""

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libmlegs_b200.so")

c_int = ctypes.c_int
c_double = ctypes.c_double
c_void_p = ctypes.c_void_p
c_int64 = ctypes.c_int64
c_char_p = ctypes.c_char_p
dptr = ctypes.POINTER(ctypes.c_double)


class Vortex(ctypes.Structure):
    """mlegs_vortex (include/mlegs_b200.h): one QPAIR entry."""
    _fields_ = [(k, ctypes.c_double) for k in ("x", "y", "q", "h", "b", "dx", "dy", "k", "dp", "r", "dr", "rk", "rp")]


class Params(ctypes.Structure):
    """mlegs_params (include/mlegs_b200.h)."""
    _fields_ = [
        ("nr", ctypes.c_int32), ("nth", ctypes.c_int32), ("nx", ctypes.c_int32),
        ("nrchop", ctypes.c_int32), ("ntchop", ctypes.c_int32), ("nxchop", ctypes.c_int32),
        ("ell", c_double), ("zlen", c_double),
        ("dt", c_double),
        ("adams", ctypes.c_int32),
        ("omega", c_double), ("bv0", c_double), ("kappa", c_double), ("kappap", c_double),
        ("visc_sw", ctypes.c_int32), ("visc_p", ctypes.c_int32),
        ("nu", c_double), ("nup", c_double),
        ("precision", ctypes.c_int32), ("split_slices", ctypes.c_int32),
        ("device", ctypes.c_int32), ("rmv_sw", ctypes.c_int32),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "mlegs_create": (c_int, [ctypes.POINTER(Params), ctypes.POINTER(c_void_p)]),
    "mlegs_destroy": (c_int, [c_void_p]),
    "mlegs_last_error": (c_char_p, [c_void_p]),
    "mlegs_sync": (c_int, [c_void_p]),
    "mlegs_set_wait_limit": (c_int, [c_void_p, c_int64]),
    "mlegs_dims": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "mlegs_field_alloc": (c_int, [c_void_p, c_int, ctypes.POINTER(c_void_p)]),
    "mlegs_field_free": (c_int, [c_void_p, c_void_p]),
    "mlegs_field_space": (c_int, [c_void_p]),
    "mlegs_field_upload": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_double]),
    "mlegs_field_download": (c_int, [c_void_p, c_void_p, c_void_p, dptr]),
    "mlegs_field_copy": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_grid": (c_int, [c_void_p, dptr, dptr, dptr]),
    "mlegs_field_axpby": (c_int, [c_void_p, c_void_p, c_double, c_void_p, c_double, c_void_p, c_double]),
    "mlegs_field_set_ln": (c_int, [c_void_p, c_void_p, c_double]),
    "mlegs_chopdo": (c_int, [c_void_p, c_void_p, c_int]),
    "mlegs_rtran": (c_int, [c_void_p, c_void_p, c_int, c_int]),
    "mlegs_horfft": (c_int, [c_void_p, c_void_p, c_int]),
    "mlegs_verfft": (c_int, [c_void_p, c_void_p, c_int]),
    "mlegs_plnfft": (c_int, [c_void_p, c_void_p, c_int]),
    "mlegs_toff": (c_int, [c_void_p, c_void_p, c_int]),
    "mlegs_tofp": (c_int, [c_void_p, c_void_p, c_int]),
    "mlegs_delsqh": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_idelsqh": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_mulxm": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_xxdx": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_del2": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_idel2": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_double, c_int]),
    "mlegs_idel2ln": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_idel2ln_static": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_ihelm": (c_int, [c_void_p, c_void_p, c_void_p, c_double, c_int]),
    "mlegs_ihelmp": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_double, c_double, c_int]),
    "mlegs_hyperv": (c_int, [c_void_p, c_void_p, c_double, c_double, c_int, c_double]),
    "mlegs_grad": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_pc2vel": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_pc2vor": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int]),
    "mlegs_project": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_double]),
    "mlegs_boussi_force": (c_int, [c_void_p] + [c_void_p] * 6),
    "mlegs_boussi_nonlin": (c_int, [c_void_p] + [c_void_p] * 8),
    "mlegs_legendre_table": (c_int, [c_void_p, c_void_p]),
    "mlegs_boussi_energy": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "mlegs_boussi_pe": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mlegs_diagnost": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mlegs_qvortex": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "mlegs_enemon": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "mlegs_hyp3adj": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mlegs_hyp3_coeffs": (c_int, [c_void_p, c_void_p]),
    "mlegs_specurv": (c_int, [c_void_p, c_int, c_double, c_void_p]),
    "mlegs_speslop": (c_int, [c_void_p, c_int, c_double, c_void_p]),
    "mlegs_pdajust": (c_int, [c_void_p, c_double, c_double, c_double, c_void_p, c_int, c_double]),
    "mlegs_hyp3_controller": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p]),
    "mlegs_msave": (c_int, [c_void_p, c_void_p, ctypes.c_char_p, c_int]),
    "mlegs_mload": (c_int, [c_void_p, ctypes.c_char_p, c_void_p, c_int]),
    "mlegs_solver_init": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mlegs_step": (c_int, [c_void_p, c_int]),
    "mlegs_step_graph": (c_int, [c_void_p, c_int]),
    "mlegs_run_host": (c_int, [c_void_p, c_int, c_void_p, dptr]),
    "mlegs_time": (c_int, [c_void_p, dptr, ctypes.POINTER(ctypes.c_int32)]),
    "mlegs_check_finite": (c_int, [c_void_p]),
    "mlegs_kernel_time": (c_int, [c_void_p, c_int, c_int, dptr, dptr]),
    "mlegs_ensemble_create": (c_int, [ctypes.POINTER(Params), c_int, ctypes.POINTER(c_void_p)]),
    "mlegs_ensemble_destroy": (c_int, [c_void_p]),
    "mlegs_ensemble_last_error": (c_char_p, [c_void_p]),
    "mlegs_ensemble_size": (c_int, [c_void_p]),
    "mlegs_ensemble_context": (c_void_p, [c_void_p, c_int]),
    "mlegs_ensemble_step": (c_int, [c_void_p, c_int, c_int]),
    "mlegs_ensemble_tune": (c_int, [c_void_p]),
    "mlegs_ensemble_tuning": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_int32), c_int]),
    "mlegs_ensemble_ctas": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "mlegs_ensemble_sync": (c_int, [c_void_p]),
    "mlegs_ensemble_launch_count": (c_int64, [c_void_p]),
    "mlegs_ensemble_stream": (c_void_p, [c_void_p]),
    "mlegs_transpose": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int, c_double]),
    "mlegs_boussi_force_vjp": (c_int, [c_void_p] + [c_void_p] * 9),
    "mlegs_ab2_step_map": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mlegs_ab2_step_vjp": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mlegs_ab2_startup_map": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mlegs_ab2_startup_vjp": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "mlegs_initial_state_T": (c_int, [c_void_p, c_void_p, c_void_p]),
    "mlegs_energy_objective": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, dptr, c_void_p, c_void_p, c_void_p]),
    "mlegs_field_device_copy": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "mlegs_launch_count": (c_int64, [c_void_p]),
    "mlegs_reset_launch_count": (None, [c_void_p]),
    "mlegs_stream": (c_void_p, [c_void_p]),
}

_LIB = None


def load(path=LIBPATH):
    """Load the shared library once and attach every declared signature."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError("libmlegs_b200.so is not built (run `python -m mlegs_b200.build`); "
                           "there is no CPU fallback")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib
