"""ctypes binding of the in-tree CUDA library (``include/dmrgpp_kron.h``).

The library is the product path: there is no fallback.  Importing this module
fails loudly if ``_lib/libdmrgpp_kron.so`` is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libdmrgpp_kron.so")

OK, INVALID_ARG, OOM, CUDA_ERROR, TIMEOUT, NOT_SUPPORTED, NOT_CONVERGED = range(7)
FP64, SPLIT_BF16, TF32X3 = 0, 1, 2
STATUS_NAMES = {OK: "OK", INVALID_ARG: "INVALID_ARG", OOM: "OOM", CUDA_ERROR: "CUDA_ERROR",
                TIMEOUT: "TIMEOUT", NOT_SUPPORTED: "NOT_SUPPORTED",
                NOT_CONVERGED: "NOT_CONVERGED"}

_sz = ctypes.c_size_t
_szp = ctypes.POINTER(ctypes.c_size_t)
_dp = ctypes.POINTER(ctypes.c_double)
_vpp = ctypes.POINTER(ctypes.c_void_p)


class KronDesc(ctypes.Structure):
    _fields_ = [("noperator", _sz), ("npatches", _sz), ("left_patch_size", _szp),
                ("right_patch_size", _szp), ("Amatrix", _vpp), ("ld_Amatrix", _szp),
                ("Bmatrix", _vpp), ("ld_Bmatrix", _szp), ("precision", ctypes.c_int),
                ("stream", ctypes.c_void_p), ("device", ctypes.c_int)]


class WftDesc(ctypes.Structure):
    _fields_ = [("np_in", _sz), ("l_in", _szp), ("r_in", _szp), ("np_out", _sz),
                ("l_out", _szp), ("r_out", _szp), ("src", ctypes.POINTER(ctypes.c_longlong)),
                ("WL", _vpp), ("ld_WL", _szp), ("WR", _vpp), ("ld_WR", _szp),
                ("trans_WL", ctypes.c_int), ("trans_WR", ctypes.c_int),
                ("stream", ctypes.c_void_p), ("device", ctypes.c_int)]


class DensityDesc(ctypes.Structure):
    _fields_ = [("npatches", _sz), ("left_patch_size", _szp), ("right_patch_size", _szp),
                ("patch_group", _szp), ("ngroups", _sz), ("group_size", _szp),
                ("side", ctypes.c_int), ("ntargets", _sz), ("psi", ctypes.c_void_p),
                ("weights", ctypes.POINTER(ctypes.c_double)), ("stream", ctypes.c_void_p),
                ("device", ctypes.c_int)]


class Crs(ctypes.Structure):
    _fields_ = [("rows", _sz), ("rowptr", ctypes.POINTER(ctypes.c_int)),
                ("colind", ctypes.POINTER(ctypes.c_int)), ("values", ctypes.POINTER(ctypes.c_double))]


class KronCrsDesc(ctypes.Structure):
    _fields_ = [("noperator", _sz), ("npatches", _sz), ("left_offset", _szp),
                ("left_patch_size", _szp), ("right_offset", _szp), ("right_patch_size", _szp),
                ("A", ctypes.POINTER(Crs)), ("B", ctypes.POINTER(Crs)),
                ("value", ctypes.POINTER(ctypes.c_double)), ("fermion", ctypes.POINTER(ctypes.c_int)),
                ("left_parity", ctypes.POINTER(ctypes.c_ubyte)), ("precision", ctypes.c_int),
                ("stream", ctypes.c_void_p), ("device", ctypes.c_int)]


class GatherIndexDesc(ctypes.Structure):
    _fields_ = [("npatches", _sz), ("patch_left", _szp), ("patch_right", _szp),
                ("left_groups", _sz), ("left_partition", _szp), ("right_groups", _sz),
                ("right_partition", _szp), ("perm_inverse", _szp), ("offset", _sz),
                ("sector_size", _sz)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("ntriples", _sz), ("dim", _sz), ("f_alg", ctypes.c_double),
                ("operator_bytes", _sz), ("bx_bytes", _sz), ("pass1_tiles", _sz),
                ("pass2_tiles", _sz)]


# every symbol include/dmrgpp_kron.h declares, with (restype, argtypes)
SIGNATURES = {
    "dmrgpp_version": (ctypes.c_char_p, []),
    "dmrgpp_kron_create": (ctypes.c_int, [ctypes.POINTER(KronDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "dmrgpp_kron_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dmrgpp_kron_apply": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int]),
    "dmrgpp_kron_dim": (ctypes.c_int, [ctypes.c_void_p, _szp]),
    "dmrgpp_kron_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "dmrgpp_kron_set_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dmrgpp_kron_get_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "dmrgpp_kron_test_stall_dependency": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dmrgpp_kron_flops": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "dmrgpp_kron_setup_profile": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_size_t]),
    "dmrgpp_release_cached_memory": (ctypes.c_int, [ctypes.c_int]),
    "dmrgpp_kron_create_complex": (ctypes.c_int, [ctypes.POINTER(KronDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "dmrgpp_kron_is_complex": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "dmrgpp_wft_create": (ctypes.c_int, [ctypes.POINTER(WftDesc), ctypes.POINTER(ctypes.c_void_p)]),
    "dmrgpp_wft_apply": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "dmrgpp_wft_dims": (ctypes.c_int, [ctypes.c_void_p, _szp, _szp]),
    "dmrgpp_wft_flops": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "dmrgpp_wft_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "dmrgpp_wft_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "dmrgpp_cached_memory": (ctypes.c_int, [ctypes.c_int, _szp, _szp]),
    "dmrgpp_kron_plan_info_get": (ctypes.c_int, [ctypes.POINTER(KronDesc),
                                                 ctypes.POINTER(PlanInfo)]),
    "dmrgpp_kron_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "dmrgpp_kron_apply_noalloc": (ctypes.c_int, [ctypes.POINTER(KronDesc), ctypes.c_void_p,
                                                 ctypes.c_void_p]),
    "dmrgpp_kron_noalloc_last_error": (ctypes.c_char_p, []),
}
NOALLOC_SCRATCH_BYTES = 16 << 20


class LanczosParams(ctypes.Structure):
    _fields_ = [("steps", _sz), ("min_steps", _sz), ("eigs_for_stop", _sz),
                ("tolerance", ctypes.c_double), ("reortho", ctypes.c_int),
                ("check_every", ctypes.c_int), ("use_graph", ctypes.c_int),
                ("residual_gap_ratio", ctypes.c_double)]


class DavidsonParams(ctypes.Structure):
    _fields_ = [("max_iterations", _sz), ("max_subspace", _sz), ("tolerance", ctypes.c_double),
                ("preconditioner", ctypes.c_int), ("mlp", ctypes.c_void_p),
                ("mixed_tolerance", ctypes.c_double), ("denominator_floor", ctypes.c_double)]


class DavidsonStats(ctypes.Structure):
    _fields_ = [("iterations", _sz), ("mixed_matvecs", _sz), ("fp64_matvecs", _sz),
                ("restarts", _sz), ("residual_norm", ctypes.c_double), ("converged", ctypes.c_int)]


class RefineStats(ctypes.Structure):
    _fields_ = [("outer_iterations", _sz), ("inner_matvecs", _sz), ("fp64_matvecs", _sz),
                ("residual_norm", ctypes.c_double), ("converged", ctypes.c_int)]


PRECOND_NONE, PRECOND_JACOBI, PRECOND_MLP = 0, 1, 2
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p

SIGNATURES.update({
    "dmrgpp_davidson_params_init": (None, [ctypes.POINTER(DavidsonParams)]),
    "dmrgpp_davidson_lowest": (ctypes.c_int, [_vp, ctypes.POINTER(DavidsonParams), _vp, ctypes.c_int,
                                              _dp, _vp, ctypes.POINTER(DavidsonStats)]),
    "dmrgpp_correction_solve": (ctypes.c_int, [_vp, _vp, ctypes.c_double, _vp, _vp, ctypes.c_int,
                                               ctypes.c_double, ctypes.POINTER(ctypes.c_int), _dp]),
    "dmrgpp_kron_diagonal": (ctypes.c_int, [_vp, _vp]),
    "dmrgpp_refine_lowest": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                            ctypes.c_double, _dp, ctypes.POINTER(RefineStats)]),
    "dmrgpp_refine_lowest_group": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_int, ctypes.c_double, _dp,
                                                  ctypes.POINTER(ctypes.c_int),
                                                  ctypes.POINTER(RefineStats)]),
    "dmrgpp_mlp_num_params": (_sz, []),
    "dmrgpp_mlp_create": (ctypes.c_int, [ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_void_p)]),
    "dmrgpp_mlp_destroy": (ctypes.c_int, [_vp]),
    "dmrgpp_mlp_get_params": (ctypes.c_int, [_vp, _fp, _sz]),
    "dmrgpp_mlp_set_params": (ctypes.c_int, [_vp, _fp, _sz]),
    "dmrgpp_mlp_get_grads": (ctypes.c_int, [_vp, _fp, _sz]),
    "dmrgpp_mlp_features": (ctypes.c_int, [_vp, _vp, ctypes.c_double, ctypes.c_double, _sz, _vp, _vp]),
    "dmrgpp_mlp_forward": (ctypes.c_int, [_vp, _vp, ctypes.c_int, _vp, _vp]),
    "dmrgpp_mlp_backward": (ctypes.c_int, [_vp, _vp, _vp, _vp, _dp, _vp]),
    "dmrgpp_mlp_adam_step": (ctypes.c_int, [_vp, ctypes.c_float, _vp]),
    "dmrgpp_mlp_set_inference": (ctypes.c_int, [_vp, ctypes.c_int]),
    "dmrgpp_mlp_precondition": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_double, ctypes.c_double, _vp,
                                               _sz, _vp]),
    "dmrgpp_mlp_precondition_group": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int,
                                                     _vp, _sz, _vp]),
    "dmrgpp_davidson_lowest_group": (ctypes.c_int, [_vp, ctypes.POINTER(DavidsonParams), _vp,
                                                    ctypes.c_int, _dp, _vp,
                                                    ctypes.POINTER(ctypes.c_int),
                                                    ctypes.POINTER(DavidsonStats)]),
    "dmrgpp_mlp_last_error": (ctypes.c_char_p, [_vp]),
    "dmrgpp_kron_create_crs": (ctypes.c_int, [ctypes.POINTER(KronCrsDesc),
                                              ctypes.POINTER(ctypes.c_void_p)]),
    "dmrgpp_density_truncate": (ctypes.c_int, [ctypes.POINTER(DensityDesc), _sz, ctypes.c_double,
                                               _sz, _dp, _dp, _szp, _szp, _dp]),
    "dmrgpp_density_profile": (ctypes.c_int, [_dp, ctypes.c_int]),
})

SIGNATURES.update({
    "dmrgpp_lanczos_params_init": (None, [ctypes.POINTER(LanczosParams)]),
    "dmrgpp_kron_create_group": (ctypes.c_int, [ctypes.POINTER(KronDesc), _sz,
                                                ctypes.POINTER(ctypes.c_void_p)]),
    "dmrgpp_kron_group_sectors": (ctypes.c_int, [ctypes.c_void_p, _szp,
                                                 ctypes.POINTER(ctypes.c_longlong)]),
    "dmrgpp_lanczos_lowest_group": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LanczosParams),
                                                   ctypes.c_void_p, ctypes.c_int, _dp,
                                                   ctypes.c_void_p, _szp]),
    "dmrgpp_lanczos_lowest_group_masked": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LanczosParams),
                                                          ctypes.c_void_p, ctypes.c_int,
                                                          ctypes.POINTER(ctypes.c_int), _dp,
                                                          ctypes.c_void_p, _szp]),
    "dmrgpp_lanczos_lowest": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(LanczosParams),
                                             ctypes.c_void_p, ctypes.c_int, _dp, ctypes.c_void_p,
                                             _szp]),
    "dmrgpp_tridiag_eigen": (ctypes.c_int, [_sz, _dp, _dp, _dp, _dp]),
    "dmrgpp_gather": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _sz,
                                     ctypes.c_void_p]),
    "dmrgpp_kron_get_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int)]),
    "dmrgpp_kron_set_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "dmrgpp_kron_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_int), _dp]),
    "dmrgpp_scatter": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _sz,
                                      ctypes.c_void_p]),
    "dmrgpp_kron_gather_index": (ctypes.c_int, [ctypes.POINTER(GatherIndexDesc),
                                                ctypes.POINTER(ctypes.c_int64)]),
    "dmrgpp_kron_tuned_times": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "dmrgpp_set_correction_preconditioner": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "dmrgpp_kron_patch_list": (ctypes.c_int, [_sz, ctypes.POINTER(ctypes.c_int64), _sz,
                                              ctypes.POINTER(ctypes.c_int64), _sz,
                                              ctypes.POINTER(ctypes.c_int64), _sz, _szp, _szp,
                                              _szp]),
})


class DmrgppError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"CUDA library {LIB_PATH} is missing; build it with "
                "`python -m dmrgpp_b200.build` (there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status, handle=None):
    if status != OK:
        msg = lib().dmrgpp_kron_last_error(handle)
        raise DmrgppError(status, msg.decode() if msg else "")
