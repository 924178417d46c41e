"""ctypes binding of the C ABI in include/flam.h.

The shared library is built in-tree (``flam_b200/libflam_b200.so``) by
``flam_b200.build``.  There is no fallback: importing a function that needs
the library raises if it is missing or was built without the device code.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libflam_b200.so")

FLAM_OK = 0
STATUS = {
    0: "FLAM_OK", 1: "FLAM_ERR_ARG", 2: "FLAM_ERR_NOT_SPD", 3: "FLAM_ERR_CUDA", 4: "FLAM_ERR_NOMEM",
    5: "FLAM_ERR_UNSUPPORTED", 6: "FLAM_ERR_TIMEOUT",
    100: "FLAM_WARN_RRQR_MAXITER", 101: "FLAM_WARN_SINGULAR", 102: "FLAM_WARN_IR_NOT_CONVERGED",
    103: "FLAM_WARN_LDL_AS_LU",
}

# every symbol include/flam.h declares
EXPORTS = (
    "flam_opts_default", "flam_hypoct", "flam_id", "flam_id_noalloc", "flam_rskelf", "flam_rskelf_batched", "flam_rskelf_sv", "flam_rskelf_mv",
    "flam_factor_info", "flam_tree_export", "flam_tree_perm", "flam_factor_sizes", "flam_factor_export",
    "flam_level_stats", "flam_factor_free", "flam_workspace_release", "flam_profile", "flam_last_error", "flam_version",
    "flam_rskelf_cholmv", "flam_rskelf_cholsv", "flam_rskelf_logdet", "flam_partial_sizes", "flam_partial_export",
    "flam_rskelf_partial_sv", "flam_rskelf_partial_mv", "flam_factor_import", "flam_rskelf_diag",
    "flam_matvec", "flam_rskelf_ir_sv", "flam_predictor_create", "flam_predictor_free", "flam_predictor_get",
    "flam_predictor_set", "flam_predictor_train", "flam_predictor_eval", "flam_predictor_grad", "flam_rank_log",
    "flam_autotune", "flam_tune_get", "flam_tune_set",
)

# int fn(double* Y, int64_t n, int64_t nrhs, char trans, void* stream, void* ctx)
SKEL_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int64, C.c_char, C.c_void_p, C.c_void_p)


class FlamKernel(C.Structure):
    _fields_ = [("kind", C.c_int), ("scale", C.c_double), ("dval", C.c_double), ("param", C.c_double),
                ("weights", C.c_void_p), ("normals", C.c_void_p)]


class FlamProxy(C.Structure):
    _fields_ = [("kind", C.c_int), ("p", C.c_int), ("p_rad", C.c_int), ("kernel_kind", C.c_int),
                ("scale", C.c_double), ("param", C.c_double), ("two_sided", C.c_int)]


class FlamOpts(C.Structure):
    _fields_ = [("lvlmax", C.c_int), ("ext", C.c_void_p), ("Tmax", C.c_double), ("rrqr_iter", C.c_int64),
                ("symm", C.c_char), ("stop", C.c_int), ("verb", C.c_int), ("stream", C.c_void_p),
                ("profile", C.c_int), ("sketch", C.c_int), ("sketch_p", C.c_int), ("sketch_guard", C.c_int),
                ("sketch_seed", C.c_uint), ("predictor", C.c_void_p), ("rank_log", C.c_int)]


class FlamTune(C.Structure):
    _fields_ = [("split_ctas", C.c_int), ("split_max", C.c_int), ("split_min_n", C.c_int), ("tc_smem_max", C.c_int)]


class FlamInfo(C.Structure):
    _fields_ = [("N", C.c_int64), ("ninst", C.c_int), ("d", C.c_int), ("symm", C.c_char), ("nbox", C.c_int64),
                ("nlvl_max", C.c_int), ("nfactor", C.c_int64), ("nstep", C.c_int), ("bytes", C.c_int64),
                ("nrem", C.c_int64), ("t_tree", C.c_double), ("t_factor", C.c_double)]


class FlamProf(C.Structure):
    _fields_ = [("launches", C.c_int64), ("n_compress", C.c_int64), ("n_elim", C.c_int64), ("n_sweep", C.c_int64),
                ("t_compress", C.c_double), ("t_elim", C.c_double), ("t_sweep", C.c_double),
                ("flop_compress", C.c_double), ("flop_elim", C.c_double), ("flop_sweep", C.c_double),
                ("byte_sweep", C.c_double), ("n_sketch", C.c_int64), ("n_sketch_redo", C.c_int64),
                ("sketch_rows", C.c_int64), ("sketch_rows_k", C.c_int64), ("id_rows", C.c_int64),
                ("graph_replays", C.c_int64), ("t_sketch", C.c_double), ("flop_sketch", C.c_double),
                ("flop_id", C.c_double)]


class FlamError(RuntimeError):
    """Error raised with the reference's identifier, e.g. ``FLAM:chksymm:invalidSymm``."""

    def __init__(self, code, msg):
        self.code = code
        self.identifier = msg.split(": ", 1)[0] if msg.startswith("FLAM:") else ""
        super().__init__(f"{STATUS.get(code, code)}: {msg}")


_lib = None


def lib():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"flam_b200: CUDA library missing at {LIB_PATH}; run `python -m flam_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    i64p = C.POINTER(C.c_int64)
    dp = C.POINTER(C.c_double)
    L.flam_opts_default.argtypes = [C.POINTER(FlamOpts)]
    L.flam_opts_default.restype = None
    L.flam_rskelf.argtypes = [P, C.c_int, C.c_int64, C.POINTER(FlamKernel), C.c_double, C.c_double,
                              C.POINTER(FlamProxy), C.POINTER(FlamOpts), C.POINTER(P)]
    L.flam_rskelf.restype = C.c_int
    L.flam_hypoct.argtypes = [P, C.c_int, C.c_int64, C.c_double, C.c_int, P, P, C.POINTER(P)]
    L.flam_hypoct.restype = C.c_int
    L.flam_id.argtypes = [P, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int64, i64p, i64p, dp,
                          i64p]
    L.flam_id.restype = C.c_int
    L.flam_id_noalloc.argtypes = [P, C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_int64, P, P, P,
                                  P, P]
    L.flam_id_noalloc.restype = C.c_int
    L.flam_rskelf_batched.argtypes = [C.c_int, P, C.c_int, i64p, C.POINTER(FlamKernel), C.c_double, C.c_double,
                                      C.POINTER(FlamProxy), C.POINTER(FlamOpts), C.POINTER(P)]
    L.flam_rskelf_batched.restype = C.c_int
    for f in ("flam_rskelf_sv", "flam_rskelf_mv", "flam_rskelf_cholmv", "flam_rskelf_cholsv"):
        getattr(L, f).argtypes = [P, P, C.c_int64, C.c_int64, C.c_char]
        getattr(L, f).restype = C.c_int
    for f in ("flam_rskelf_partial_sv", "flam_rskelf_partial_mv"):
        getattr(L, f).argtypes = [P, P, C.c_int64, C.c_int64, C.c_char, SKEL_FN, P]
        getattr(L, f).restype = C.c_int
    L.flam_factor_import.argtypes = [C.c_int64, C.c_char, C.c_int64, i64p, i64p, i64p, i64p, dp, dp, dp, i64p, dp,
                                     dp, P, C.POINTER(P)]
    L.flam_factor_import.restype = C.c_int
    L.flam_matvec.argtypes = [P, P, C.c_int64, C.c_int64, P, C.c_int64, P, C.c_int64]
    L.flam_matvec.restype = C.c_int
    L.flam_rskelf_ir_sv.argtypes = [P, P, C.c_int64, P, C.c_int64, C.c_int64, C.c_double, C.c_int,
                                    C.POINTER(C.c_int), dp]
    L.flam_rskelf_ir_sv.restype = C.c_int
    fp = C.POINTER(C.c_float)
    L.flam_predictor_create.argtypes = [C.c_uint64, C.POINTER(P)]
    L.flam_predictor_create.restype = C.c_int
    L.flam_predictor_free.argtypes = [P]
    L.flam_predictor_free.restype = None
    L.flam_predictor_get.argtypes = [P, fp]
    L.flam_predictor_get.restype = C.c_int
    L.flam_predictor_set.argtypes = [P, fp]
    L.flam_predictor_set.restype = C.c_int
    L.flam_predictor_train.argtypes = [P, fp, fp, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64, fp]
    L.flam_predictor_train.restype = C.c_int
    L.flam_predictor_eval.argtypes = [P, fp, C.c_int64, fp]
    L.flam_predictor_eval.restype = C.c_int
    L.flam_predictor_grad.argtypes = [P, fp, fp, C.c_int64, fp, fp]
    L.flam_predictor_grad.restype = C.c_int
    L.flam_rank_log.argtypes = [P, C.POINTER(C.c_int64), fp, fp]
    L.flam_rank_log.restype = C.c_int
    L.flam_autotune.argtypes = [P, C.c_int, C.c_int64, C.POINTER(FlamKernel), C.c_double, C.c_double,
                                C.POINTER(FlamProxy), C.POINTER(FlamOpts), C.c_int, C.POINTER(FlamTune)]
    L.flam_autotune.restype = C.c_int
    L.flam_tune_get.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(FlamTune)]
    L.flam_tune_get.restype = C.c_int
    L.flam_tune_set.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(FlamTune)]
    L.flam_tune_set.restype = C.c_int
    L.flam_rskelf_diag.argtypes = [P, C.c_int, P]
    L.flam_rskelf_diag.restype = C.c_int
    L.flam_rskelf_logdet.argtypes = [P, dp, dp]
    L.flam_rskelf_logdet.restype = C.c_int
    L.flam_partial_sizes.argtypes = [P, C.c_int, i64p, i64p]
    L.flam_partial_sizes.restype = C.c_int
    L.flam_partial_export.argtypes = [P, C.c_int, i64p, i64p, i64p, dp]
    L.flam_partial_export.restype = C.c_int
    L.flam_factor_info.argtypes = [P, C.POINTER(FlamInfo)]
    L.flam_factor_info.restype = C.c_int
    L.flam_tree_export.argtypes = [P, C.c_int, C.POINTER(C.c_int), i64p, i64p, i64p, i64p, i64p, dp, dp, i64p,
                                   i64p, i64p, i64p, i64p, i64p, i64p]
    L.flam_tree_export.restype = C.c_int
    L.flam_tree_perm.argtypes = [P, C.c_int, i64p]
    L.flam_tree_perm.restype = C.c_int
    L.flam_factor_sizes.argtypes = [P, C.c_int, i64p, C.POINTER(C.c_int), i64p, i64p, i64p]
    L.flam_factor_sizes.restype = C.c_int
    L.flam_factor_export.argtypes = [P, C.c_int, C.c_int64, i64p, i64p, dp, dp, dp, i64p, dp, dp]
    L.flam_factor_export.restype = C.c_int
    L.flam_level_stats.argtypes = [P, C.c_int, C.POINTER(C.c_int), i64p]
    L.flam_level_stats.restype = C.c_int
    L.flam_profile.argtypes = [P, C.POINTER(FlamProf), C.c_int]
    L.flam_profile.restype = C.c_int
    L.flam_workspace_release.argtypes = []
    L.flam_workspace_release.restype = None
    L.flam_factor_free.argtypes = [P]
    L.flam_factor_free.restype = None
    L.flam_last_error.argtypes = []
    L.flam_last_error.restype = C.c_char_p
    L.flam_version.argtypes = []
    L.flam_version.restype = C.c_char_p
    _lib = L
    return L


def check(code, allow_warn=True):
    if code == FLAM_OK:
        return code
    msg = lib().flam_last_error().decode()
    if allow_warn and code >= 100:
        import warnings
        warnings.warn(msg)
        return code
    raise FlamError(code, msg)
