"""ctypes binding of libgrimgpu.so (the C ABI declared in include/grimgpu.h).

The product path has no CPU fallback: if the library is missing or the CUDA device
is unusable, every entry point raises ``GrimError``.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libgrimgpu.so')

GRIM_OK = 0
GRIM_ERR_ARGUMENT = 3
GRIM_ERR_CUDA = 4
GRIM_ERR_NOMEM = 5
GRIM_ERR_SINGULAR = 6
GRIM_ERR_NOT_CONVERGED = 7
GRIM_ERR_NONFINITE = 8
POL_TM, POL_TE = 0, 1
PREC_FP64, PREC_MIXED, PREC_MIXED_BERR = 0, 1, 2
PREC_STATIC_PIVOT, PREC_PARTIAL_PIVOT, PREC_TOURNAMENT_PIVOT = 8, 16, 32
PIVOT_CERTIFIED, PIVOT_STATIC, PIVOT_PARTIAL, PIVOT_TOURNAMENT = 0, 1, 2, 3
TUNE_SOLVE_BN, TUNE_GS_BLOCK, TUNE_PIVOT = 1, 2, 3

c_int, c_int64, c_double, c_void_p, c_char_p = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p, ctypes.c_char_p
c_size_t = ctypes.c_size_t
P_int = ctypes.POINTER(ctypes.c_int)


class GrimCondSystem(ctypes.Structure):
    """``grim_cond_system`` of include/grimgpu.h (one factored system for grim_zcond1_factored)."""
    _fields_ = [('n', c_int), ('A', c_void_p), ('lda', c_int64), ('halves', c_int), ('lu_complex64', c_int),
                ('lu', c_void_p * 2), ('ldlu', c_int64 * 2), ('ipiv', c_void_p * 2), ('k', c_int), ('nfe', c_int),
                ('nfo', c_int), ('p1', c_void_p), ('p2', c_void_p), ('fe', c_void_p), ('fo', c_void_p),
                ('s', c_void_p)]


class GrimSolveInfo(ctypes.Structure):
    _fields_ = [('backward_error', c_double), ('initial_backward_error', c_double), ('refinement_steps', c_int),
                ('pivoted_panels', c_int), ('precision_mode', c_int), ('info', c_int), ('ms_factor', c_double),
                ('ms_solve', c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class GrimError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


class GrimMemoryError(GrimError, MemoryError):
    pass


class GrimNotConverged(GrimError):
    pass


# (name, restype, argtypes) for every symbol of include/grimgpu.h
SIGNATURES = [
    ('grim_create', c_int, [c_int, ctypes.POINTER(c_void_p)]),
    ('grim_destroy', c_int, [c_void_p]),
    ('grim_set_stream', c_int, [c_void_p, c_void_p]),
    ('grim_get_stream', c_void_p, [c_void_p]),
    ('grim_synchronize', c_int, [c_void_p]),
    ('grim_last_error', c_char_p, []),
    ('grim_device_name', c_int, [c_void_p, c_char_p, c_int]),
    ('grim_version', c_int, []),
    ('grim_launch_count', c_int64, [c_void_p]),
    ('grim_release_workspace', c_int, [c_void_p]),
    ('grim_fill2d', c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_double, c_void_p, c_int64, c_int]),
    ('grim_rhs2d', c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_double, c_void_p, c_int64, c_int]),
    ('grim_farfield2d', c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_double, c_void_p, c_int64, c_int, c_void_p]),
    ('grim_gal_near_count', c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, P_int]),
    ('grim_gal_near_list', c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('grim_gal_fill', c_int, [c_void_p, c_int, c_int, c_int] + [c_void_p] * 7 + [c_int, c_void_p, c_int, c_double,
                                                                                  c_int, c_void_p, c_int64, c_int]),
    ('grim_gal_status', c_int, [c_void_p, P_int]),
    ('grim_gal_rhs', c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_double,
                             c_void_p, c_int64, c_int]),
    ('grim_gal_farfield', c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_double, c_void_p, c_int64,
                                  c_int, c_void_p]),
    ('grim_zgetrf', c_int, [c_void_p, c_int, c_void_p, c_int64, c_void_p, P_int]),
    ('grim_zgetrs', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_void_p, c_int64]),
    ('grim_cgetrf', c_int, [c_void_p, c_int, c_void_p, c_int64, c_void_p, P_int]),
    ('grim_cgetrs', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_void_p, c_int64]),
    ('grim_backward_error', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_int, c_void_p, c_int64, c_void_p,
                                    c_int64, c_void_p]),
    ('grim_cgemm_sub', c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                               c_int64, c_int]),
    ('grim_residual', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_int, c_void_p, c_int64, c_void_p, c_int64,
                              c_void_p, c_int64, c_int]),
    ('grim_zcond1_factored', c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    ('grim_solution_errors', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64,
                                     c_void_p, c_int64, c_int, c_void_p, c_void_p, c_void_p]),
    ('grim_backward_error_noalloc', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_int, c_void_p, c_int64,
                                            c_void_p, c_int64, c_void_p]),
    ('grim_zgesv_mixed', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p, c_int64,
                                 c_int, c_double, c_int, P_int, ctypes.POINTER(GrimSolveInfo)]),
    ('grim_zgesv_guarded', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_int, c_double,
                                   c_int, c_void_p, P_int, ctypes.POINTER(GrimSolveInfo)]),
    ('grim_zcond1_equilibrated', c_int, [c_void_p, c_int, c_void_p, c_int64, ctypes.POINTER(c_double)]),
    ('grim_zgesv_mixed_factored', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                          c_void_p, c_void_p, c_int64, c_double, c_int, ctypes.POINTER(GrimSolveInfo)]),
    ('grim_zgesv_refine_factored', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p,
                                           c_void_p, c_void_p, c_int64, c_int, c_double, c_int,
                                           ctypes.POINTER(GrimSolveInfo)]),
    ('grim_getrf_grouped', c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, P_int,
                                   P_int]),
    ('ghost_far_block', c_int, [c_int64, c_int64, c_int, c_int] + [c_void_p] * 7 + [c_int] * 4 +
     [c_double, c_double, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('grim_far_block', c_int, [c_void_p, c_int64, c_int64, c_int, c_int] + [c_void_p] * 7 + [c_int] * 4 +
     [c_double, c_double, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_void_p]),
    ('grim_zgesv_batched', c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_int, P_int]),
    ('grim_last_solve_info', c_int, [c_void_p, ctypes.POINTER(GrimSolveInfo)]),
    ('grim_mem_info', c_int, [c_void_p, ctypes.POINTER(c_size_t), ctypes.POINTER(c_size_t)]),
    ('grim_set_tuning', c_int, [c_void_p, c_int, c_int]),
    ('grim_bor_moments_size', c_int64, [c_int, c_int]),
    ('grim_bor_mfie_moments_size', c_int64, [c_int, c_int]),
    ('grim_bor_moments', c_int, [c_void_p, c_int, c_void_p, c_double, c_int, c_int, c_void_p, c_int, c_void_p,
                                 c_void_p, c_void_p, c_void_p]),
    ('grim_bor_assemble', c_int, [c_void_p, c_int, c_void_p, c_double, c_int, c_int, c_void_p, c_void_p, c_double,
                                  c_int, c_void_p, c_void_p, c_void_p, c_int64]),
    ('grim_bor_excitation', c_int, [c_void_p, c_int, c_void_p, c_double, c_int, c_int, c_void_p, c_int, c_double,
                                    c_int, c_void_p, c_void_p, c_void_p, c_int64]),
    ('grim_bor_mirror_halves', c_int, [c_void_p, c_int, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_void_p,
                                       c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    ('grim_bor_mirror_asymmetry', c_int, [c_void_p, c_int, c_void_p, c_int64, c_void_p, c_void_p, c_void_p]),
    ('grim_bor_mirror_split', c_int, [c_void_p, c_int, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                      c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    ('grim_bor_mirror_join', c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                     c_void_p, c_int, c_void_p, c_void_p, c_int64]),
    ('grim_bor_farfield_accumulate', c_int, [c_void_p, c_int, c_int, c_void_p, c_int64, c_void_p, c_int64, c_void_p]),
    ('grim_profile_enable', c_int, [c_void_p, c_int]),
    ('grim_profile_report', c_int, [c_void_p, c_char_p, c_int]),
]

_lib = None
_lock = threading.Lock()


def header_symbols():
    """Every function name declared in include/grimgpu.h (for export checks)."""
    import re
    path = os.path.join(os.path.dirname(_HERE), 'include', 'grimgpu.h')
    text = open(path).read()
    return sorted(set(re.findall(r'\b(grim_[a-z0-9_]+)\s*\(', text)))


def load():
    """Load libgrimgpu.so (no GPU needed) and bind every declared symbol."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise GrimError(GRIM_ERR_CUDA, f'libgrimgpu.so not built at {LIB_PATH}; run grim_20261007_b200/csrc/build.py')
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def last_error():
    msg = load().grim_last_error()
    return msg.decode(errors='replace') if msg else ''


def check(status, what=''):
    if status == GRIM_OK:
        return
    msg = f'{what}: {last_error()}' if what else last_error()
    if status == GRIM_ERR_NOMEM:
        raise GrimMemoryError(status, msg)
    if status == GRIM_ERR_NOT_CONVERGED:
        raise GrimNotConverged(status, msg)
    raise GrimError(status, msg)
