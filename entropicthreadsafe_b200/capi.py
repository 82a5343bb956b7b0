"""ctypes binding of the C-ABI declared in include/tslb.h (libtslb.so).

This is the Python side of the same boundary a Fortran host binds with
iso_c_binding; every function maps 1:1 onto an `extern "C"` entry point.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtslb.so")

# ---- constants mirrored from include/tslb.h ----
OK, ERR_ARG, ERR_CUDA, ERR_NAN, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_STATE = range(7)
MODE_PHASEFIELD, MODE_COLOUR, MODE_SINGLE = 0, 1, 2
PREC_FP32, PREC_BF16, PREC_FP16S = 0, 1, 2
BC_PERIODIC, BC_BOUNCEBACK, BC_VELOCITY, BC_INLET, BC_OUTLET, BC_PRESSURE = range(6)
MBC_NONE, MBC_COPY, MBC_JET = range(3)
FACE_XM, FACE_XP, FACE_YM, FACE_YP, FACE_ZM, FACE_ZP = range(6)
NREDUCE = 12
NOALLOC_SCRATCH_WORDS = 64
REDUCE_QUEUE = 256
RED_NAMES = ("mass", "mass_a", "mass_b", "mom_x", "mom_y", "mom_z", "kinetic",
             "umax", "rho_in", "rho_out", "dp", "n_in")
FIELDS = ("rho", "u", "v", "w", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz", "phi")


class TslbParams(ctypes.Structure):
    """Mirror of `tslb_params` (include/tslb.h)."""

    _fields_ = [
        ("mode", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("tau_a", ctypes.c_float),
        ("tau_b", ctypes.c_float),
        ("sigma", ctypes.c_float),
        ("beta", ctypes.c_float),
        ("sharp_c", ctypes.c_float),
        ("grad_threshold", ctypes.c_float),
        ("force", ctypes.c_float * 3),
        ("bc", ctypes.c_int32 * 6),
        ("bc_u", (ctypes.c_float * 3) * 6),
        ("bc_phi", ctypes.c_float * 6),
        ("wall_phi_mode", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 7),
    ]


def default_params() -> TslbParams:
    """Python restatement of tslb_default_params (no library needed)."""
    p = TslbParams()
    p.mode = MODE_PHASEFIELD
    p.precision = PREC_FP32
    p.tau_a = 0.5004
    p.tau_b = 0.5004
    p.sigma = 0.001
    p.beta = 0.7
    p.sharp_c = float(np.float32(0.3) * np.float32(3))  # single-precision 0.3*3 of the reference
    p.grad_threshold = 1e-3
    for f in range(6):
        p.bc[f] = BC_PERIODIC
        p.bc_phi[f] = 0.0
    p.wall_phi_mode = 0
    return p


def make_params(**kw) -> TslbParams:
    """default_params() with fields overridden by keyword (force/bc/bc_u/bc_phi as sequences)."""
    p = default_params()
    for k, v in kw.items():
        if k == "force":
            for a in range(3):
                p.force[a] = float(v[a])
        elif k == "bc":
            for f in range(6):
                p.bc[f] = int(v[f])
        elif k == "bc_u":
            for f in range(6):
                for a in range(3):
                    p.bc_u[f][a] = float(v[f][a])
        elif k == "bc_phi":
            for f in range(6):
                p.bc_phi[f] = float(v[f])
        else:
            setattr(p, k, v)
    return p


# learned closure (include/tslb_closure.h)
CLOSURE_NFEAT = 10
CLOSURE_HIDDEN = 64
CLOSURE_OFF = {"W1": 0, "b1": 1024, "W2": 1088, "b2": 5184, "w3": 5248, "b3": 5312}
CLOSURE_NPARAM = 5313


def _declare_closure(L) -> None:
    vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)
    ll, dp = ctypes.c_longlong, ctypes.POINTER(ctypes.c_double)
    sig = {
        "tslb_closure_create": ([ctypes.POINTER(vp)], ip),
        "tslb_closure_destroy": ([vp], None),
        "tslb_closure_set_params": ([vp, fp, fp, fp, ctypes.c_float], ip),
        "tslb_closure_get_params": ([vp, fp, fp, fp, fp], ip),
        "tslb_closure_set_dtau_min": ([vp, ctypes.c_float], ip),
        "tslb_closure_dtau_min": ([vp], ctypes.c_float),
        "tslb_closure_forward": ([vp, fp, ll, fp], ip),
        "tslb_closure_gradient": ([vp, fp, fp, fp, ll, fp, dp], ip),
        "tslb_closure_dataset_clear": ([vp], ip),
        "tslb_closure_dataset_add": ([vp, fp, fp, fp, ll], ip),
        "tslb_closure_dataset_add_fine": ([vp, vp, ctypes.c_float, ip, ip, ip, ctypes.POINTER(ll)], ip),
        "tslb_closure_dataset_size": ([vp], ll),
        "tslb_closure_dataset_download": ([vp, fp, fp, fp], ip),
        "tslb_closure_normalize": ([vp], ip),
        "tslb_closure_train": ([vp, ip, ip, ctypes.c_float, ctypes.c_ulonglong, fp], ip),
        "tslb_closure_features": ([vp, vp, fp], ip),
        "tslb_attach_closure": ([vp, vp, ip], ip),
        "tslb_closure_last_error": ([vp], ctypes.c_char_p),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res


_lib = None


def lib() -> ctypes.CDLL:
    """Load libtslb.so (built in-tree by entropicthreadsafe_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with entropicthreadsafe_b200.build.build()")
        L = ctypes.CDLL(LIB_PATH)
        vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float)
        dp = ctypes.POINTER(ctypes.c_double)
        L.tslb_default_params.argtypes = [vp]
        L.tslb_default_params.restype = None
        L.tslb_create.argtypes = [vp, ip, ip, ip, ctypes.POINTER(vp)]
        L.tslb_create.restype = ip
        L.tslb_destroy.argtypes = [vp]
        L.tslb_destroy.restype = None
        L.tslb_upload_moments.argtypes = [vp] + [fp] * 11
        L.tslb_upload_moments.restype = ip
        L.tslb_upload_pops.argtypes = [vp, fp, fp]
        L.tslb_upload_pops.restype = ip
        L.tslb_step.argtypes = [vp, ip]
        L.tslb_step.restype = ip
        L.tslb_download_moments.argtypes = [vp] + [fp] * 11
        L.tslb_download_moments.restype = ip
        L.tslb_download_normals.argtypes = [vp, fp, fp, fp]
        L.tslb_download_normals.restype = ip
        L.tslb_reduce.argtypes = [vp, dp]
        L.tslb_reduce.restype = ip
        L.tslb_set_inlet.argtypes = [vp, ip, fp]
        L.tslb_set_inlet.restype = ip
        L.tslb_synchronize.argtypes = [vp]
        L.tslb_synchronize.restype = ip
        L.tslb_stream.argtypes = [vp]
        L.tslb_stream.restype = vp
        L.tslb_launch_count.argtypes = [vp]
        L.tslb_launch_count.restype = ctypes.c_longlong
        L.tslb_last_error.argtypes = [vp]
        L.tslb_last_error.restype = ctypes.c_char_p
        L.tslb_step_noalloc.argtypes = [vp, ip, ip, ip, vp, vp, ctypes.c_longlong, vp]
        L.tslb_step_noalloc.restype = ip
        L.tslb_noalloc_check.argtypes = [vp]
        L.tslb_noalloc_check.restype = ip
        L.tslb_reduce_async.argtypes = [vp]
        L.tslb_reduce_async.restype = ip
        L.tslb_reduce_collect.argtypes = [vp, dp, ip, ctypes.POINTER(ctypes.c_int)]
        L.tslb_reduce_collect.restype = ip
        L.tslb_create_slab.argtypes = [vp, ip, ip, ip, ip, ip, ctypes.POINTER(vp)]
        L.tslb_create_slab.restype = ip
        L.tslb_slab_geometry.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
        L.tslb_slab_geometry.restype = ip
        L.tslb_halo_bytes.argtypes = [vp]
        L.tslb_halo_bytes.restype = ctypes.c_longlong
        L.tslb_halo_pack.argtypes = [vp, ip, vp]
        L.tslb_halo_pack.restype = ip
        L.tslb_halo_unpack.argtypes = [vp, ip, vp]
        L.tslb_halo_unpack.restype = ip
        L.tslb_ensemble_create.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ip, ctypes.POINTER(vp)]
        L.tslb_ensemble_create.restype = ip
        L.tslb_ensemble_destroy.argtypes = [vp]
        L.tslb_ensemble_destroy.restype = None
        L.tslb_ensemble_upload_moments.argtypes = [vp, ip] + [fp] * 11
        L.tslb_ensemble_upload_moments.restype = ip
        L.tslb_ensemble_download_moments.argtypes = [vp, ip] + [fp] * 11
        L.tslb_ensemble_download_moments.restype = ip
        L.tslb_ensemble_step.argtypes = [vp, ip]
        L.tslb_ensemble_step.restype = ip
        L.tslb_ensemble_step_graph.argtypes = [vp, ip]
        L.tslb_ensemble_step_graph.restype = ip
        L.tslb_ensemble_reduce.argtypes = [vp, ip, dp]
        L.tslb_ensemble_reduce.restype = ip
        L.tslb_ensemble_tune.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.tslb_ensemble_tune.restype = ip
        ipp = ctypes.POINTER(ctypes.c_int)
        L.tslb_ensemble_tune_results.argtypes = [vp, ip, ipp, ipp, ipp, ctypes.POINTER(ctypes.c_float)]
        L.tslb_ensemble_tune_results.restype = ip
        L.tslb_ensemble_set_launch.argtypes = [vp, ip, ip]
        L.tslb_ensemble_set_launch.restype = ip
        L.tslb_ensemble_synchronize.argtypes = [vp]
        L.tslb_ensemble_synchronize.restype = ip
        L.tslb_ensemble_stream.argtypes = [vp]
        L.tslb_ensemble_stream.restype = vp
        L.tslb_ensemble_last_error.argtypes = [vp]
        L.tslb_ensemble_last_error.restype = ctypes.c_char_p
        lp = ctypes.POINTER(ctypes.c_longlong)
        L.tslb_set_inlet_disc.argtypes = [vp, ip] + [ctypes.c_float] * 5 + [ctypes.c_ulonglong] * 2
        L.tslb_set_inlet_disc.restype = ip
        L.tslb_set_moment_bc.argtypes = [vp, ip, ip, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.tslb_set_moment_bc.restype = ip
        L.tslb_rand_noseeded.argtypes = [ip, ip, ip, ip]
        L.tslb_rand_noseeded.restype = ctypes.c_float
        L.tslb_set_solid_mask.argtypes = [vp, vp]
        L.tslb_set_solid_mask.restype = ip
        L.tslb_set_tau_correction.argtypes = [vp, fp]
        L.tslb_set_tau_correction.restype = ip
        L.tslb_download_tau_correction.argtypes = [vp, fp]
        L.tslb_download_tau_correction.restype = ip
        L.tslb_stats_reset.argtypes = [vp]
        L.tslb_stats_reset.restype = ip
        L.tslb_stats_accumulate.argtypes = [vp]
        L.tslb_stats_accumulate.restype = ip
        L.tslb_stats_download.argtypes = [vp, ip, fp, fp, fp, fp, fp, lp]
        L.tslb_stats_download.restype = ip
        L.tslb_stats_download_stress.argtypes = [vp, ip, fp, fp, lp]
        L.tslb_stats_download_stress.restype = ip
        _declare_closure(L)
        cp = ctypes.c_char_p
        for name, args, res in (("tslb_write_raw", [cp, fp, ctypes.c_longlong], ip),
                                ("tslb_write_vti", [cp, cp, ip, ip, ip, ip, fp], ip),
                                ("tslb_write_slices", [cp, cp, ip, ip, ip, ip, fp], ip),
                                ("tslb_frame_path", [ctypes.c_char_p, ip, cp, cp, cp, ip, cp], ip),
                                ("tslb_checkpoint_save", [vp, cp], ip),
                                ("tslb_checkpoint_load", [vp, cp], ip),
                                ("tslb_steps_done", [vp], ctypes.c_longlong),
                                ("tslb_host_alloc", [ctypes.c_longlong], vp),
                                ("tslb_host_free", [vp], None),
                                ("tslb_release_memory", [], ip)):
            getattr(L, name).argtypes = args
            getattr(L, name).restype = res
        _lib = L
    return _lib


DRIVER_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tslb_run")


def fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
