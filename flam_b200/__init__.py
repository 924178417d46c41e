"""flam_b200: FLAM's recursive skeletonization factorization (rskelf) on B200.

Device code: ``flam_b200/csrc`` (sm_100a CUDA), exported through the C ABI of
``include/flam.h`` as ``flam_b200/libflam_b200.so``.  This package is the
host-side mirror of the reference's MATLAB entry points.
"""
from ._lib import FlamError, lib
from .api import (Factor, Predictor, autotune, factor_import, hypoct, hypoct_perm, id, matvec, rskelf, rskelf_batched, rskelf_cholmv,
                  rskelf_cholsv, rskelf_diag, rskelf_ir_sv, rskelf_logdet, rskelf_mv, rskelf_partial_info,
                  rskelf_partial_mv, rskelf_partial_sv, rskelf_spdiag, rskelf_sv, tune_get, tune_set)
from .registry import Kernel, Proxy
from . import problems, shard

__all__ = ["FlamError", "lib", "Factor", "Predictor", "autotune", "tune_get", "tune_set", "hypoct", "hypoct_perm", "id", "rskelf", "rskelf_batched", "rskelf_mv",
           "rskelf_sv", "rskelf_cholmv", "rskelf_cholsv", "rskelf_logdet", "rskelf_partial_info",
           "rskelf_partial_sv", "rskelf_partial_mv", "rskelf_diag", "rskelf_spdiag", "factor_import", "matvec", "rskelf_ir_sv", "Kernel", "Proxy", "problems", "shard"]
