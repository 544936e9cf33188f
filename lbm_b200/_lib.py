"""ctypes binding of the C ABI in include/lbm_b200.h.

Loading fails loudly when ``liblbmb200.so`` is missing: there is no CPU or
pure-PyTorch fallback for any entry point.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbmb200.so")

LBM_OK = 0
LBM_ERR_ARG = -1
LBM_ERR_UNSUPPORTED = -2
LBM_ERR_CUDA = -3
LBM_ERR_STATE = -4
LBM_ERR_NUMERIC = -5
LBM_ERR_OOM = -6
ERR_NAMES = {0: "LBM_OK", -1: "LBM_ERR_ARG", -2: "LBM_ERR_UNSUPPORTED", -3: "LBM_ERR_CUDA",
             -4: "LBM_ERR_STATE", -5: "LBM_ERR_NUMERIC", -6: "LBM_ERR_OOM"}

LBM_STORE_F32 = 0
LBM_STORE_F16 = 1
LBM_STATUS_BAD_DENSITY = 1
LBM_STATUS_TIMEOUT = 4
LBM_KERNEL_PULL = 1
LBM_KERNEL_PAIR = 2
LBM_ENS_VARIANTS = 8
LBM_ENS_GRAPH_STEPS = 16


class LbmParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32), ("nl", ctypes.c_int32),
        ("ibgk", ctypes.c_int32), ("ihrr", ctypes.c_int32), ("ivreman", ctypes.c_int32),
        ("ibnd", ctypes.c_int32), ("jbnd", ctypes.c_int32), ("kbnd", ctypes.c_int32),
        ("iturb_pos", ctypes.c_int32), ("storage", ctypes.c_int32),
        ("kinevisc", ctypes.c_float), ("smagorinsky", ctypes.c_float), ("rho0", ctypes.c_float),
        ("udir", ctypes.c_float),
    ]


P = ctypes.c_void_p
I = ctypes.c_int32
F = ctypes.c_float
D = ctypes.c_double

# name -> argument types (all return int32 status except lbm_last_error)
SIGNATURES = {
    "lbm_create": [ctypes.POINTER(P), ctypes.POINTER(LbmParams)],
    "lbm_destroy": [P],
    "lbm_abi_version": [],
    "lbm_set_stream": [P, P],
    "lbm_synchronize": [P],
    "lbm_fequil3": [P, P, P, P, P, P],
    "lbm_postcoll": [P, P, P, P, P, P, P, P],
    "lbm_drift": [P, P, P],
    "lbm_macrovars": [P, P, P, P, P, P],
    "lbm_regularization": [P, P, P, P, P, P],
    "lbm_vreman": [P, P, P],
    "lbm_compute_fneq": [P, P, P],
    "lbm_compute_f": [P, P, P],
    "lbm_boundarycond": [P, P, P, P],
    "lbm_solids": [P, P, P],
    "lbm_inflow_turbulence_forcing": [P, P, P, P, P, P, P, P, P, F, I, I],
    "lbm_inflow_turbulence_apply": [P, P, P],
    "lbm_fillghosts": [P, P],
    # the DP build's per-call entry points: the same arguments with double arrays
    "lbm_set_params_f64": [P, D, D, D, D],
    "lbm_fequil3_f64": [P, P, P, P, P, P],
    "lbm_postcoll_f64": [P, P, P, P, P, P, P, P],
    "lbm_drift_f64": [P, P, P],
    "lbm_macrovars_f64": [P, P, P, P, P, P],
    "lbm_regularization_f64": [P, P, P, P, P, P],
    "lbm_vreman_f64": [P, P, P],
    "lbm_compute_fneq_f64": [P, P, P],
    "lbm_compute_f_f64": [P, P, P],
    "lbm_boundarycond_f64": [P, P, P, P],
    "lbm_forcings_apply_f64": [P, P, P, P, P, P, P],
    "lbm_solids_f64": [P, P, P],
    "lbm_inflow_turbulence_forcing_f64": [P, P, P, P, P, P, P, P, P, D, I, I],
    "lbm_inflow_turbulence_apply_f64": [P, P, P],
    "lbm_fillghosts_f64": [P, P],
    "lbm_state_import": [P, P, P, P, P, P, P, I],
    "lbm_state_export": [P, P, P],
    "lbm_get_macro": [P, P, P, P, P],
    "lbm_set_solids": [P, P],
    "lbm_set_turbulence": [P, P, P, P, I, F],
    "lbm_set_inflow": [P, P],
    "lbm_set_forcing": [P, P],
    "lbm_forcings_apply": [P, P, P, P, P, P, P],
    "lbm_step": [P, I],
    "lbm_step_to": [P, P],
    "lbm_set_halo_j": [P, I],
    "lbm_halo_plane_bytes": [P, P],
    "lbm_halo_pack_j": [P, P, P],
    "lbm_halo_unpack_j": [P, P, P],
    "lbm_state_snapshot_bytes": [P, P],
    "lbm_state_snapshot": [P, P],
    "lbm_state_restore": [P, P],
    "lbm_set_kernel": [P, I],
    "lbm_step_host": [P, I, P, ctypes.POINTER(ctypes.c_int32)],
    "lbm_get_step": [P, ctypes.POINTER(ctypes.c_int32)],
    "lbm_status": [P, ctypes.POINTER(ctypes.c_int32)],
    "lbm_mass_momentum": [P, P, P],
    "lbm_conservation": [P, ctypes.POINTER(ctypes.c_double)],
    "lbm_mass_momentum_noalloc": [P, I, I, I, I, P, P],
    "lbm_launch_count": [P, ctypes.POINTER(ctypes.c_int64)],
    "lbm_profile": [P, I],
    "lbm_profile_read": [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)],
    "lbm_profile_read_boundary": [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)],
    "lbm_inflow_turbulence_compute": [P, P, P, P, P, I, ctypes.c_uint64],
    "lbm_postcoll_adj": [P, P, P, P, P, P, P, P, P, P, P, P, P, P],
    "lbm_macrovars_adj": [P, P, P, P, P, P, P],
    "lbm_drift_adj": [P, P, P],
    "lbm_macrovars_drift_adj": [P, P, P, P, P, P, P, P, P, P, P],
    "lbm_boundarycond_adj": [P, P, P, P],
    "lbm_state_bytes": [P, ctypes.POINTER(ctypes.c_int64)],
    "lbm_state_copy": [P, P],
    "lbm_state_adjoint_step": [P, P, P, P, I, P],
    "lbm_state_adjoint_seed": [P, P, P, P, P, I],
    "lbm_state_adjoint_export": [P, P, P],
    "lbm_ensemble_create": [ctypes.POINTER(P), ctypes.POINTER(LbmParams), I],
    "lbm_ensemble_destroy": [P],
    "lbm_ensemble_size": [P, ctypes.POINTER(ctypes.c_int32)],
    "lbm_ensemble_member": [P, I, ctypes.POINTER(P)],
    "lbm_ensemble_step": [P, I],
    "lbm_ensemble_autotune": [P, I, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)],
    "lbm_ensemble_set_variant": [P, I],
    "lbm_ensemble_get_config": [P, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
    "lbm_ensemble_variant_shape": [I, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_int32)],
    "lbm_ensemble_profile": [P, I, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "lbm_ensemble_set_graph": [P, I],
}

_lib = None


def load():
    """Load liblbmb200.so and declare every prototype of include/lbm_b200.h."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("lbm_b200: %s is missing; build it with `python -m lbm_b200.build` "
                           "(there is no CPU fallback)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int32
    lib.lbm_last_error.argtypes = [P]
    lib.lbm_last_error.restype = ctypes.c_char_p
    lib.lbm_ensemble_last_error.argtypes = [P]
    lib.lbm_ensemble_last_error.restype = ctypes.c_char_p
    _lib = lib
    return lib


class LbmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERR_NAMES.get(code, "?"), code, msg))
        self.code = code
