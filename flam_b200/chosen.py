"""The chosen form of rskelf factor + solve to a target FP64 relative residual.

Two ways reach ``tol`` (1e-10) in FP64 on the same problem:

* plain FP64 -- the reference's algorithm (rskelf.m with id.m's exact ID of every box
  at ``tol``) followed by rskelf_sv;
* the chosen form -- the sketched factorization with learned sketch widths, in one of
  two precisions picked per problem by :func:`choose`:

  - ``"fp64-sketch"``: each box's row sketch Y = Omega K formed with FP64 entries on the
    FP64 tensor path (``opts["sketch"] = 2``), its width from the rank predictor, the
    FP64 pivoted QR, rank (at tol / 10) and R11 \\ R12 on Y.  The factorization meets
    ``tol`` itself, so the solve is one rskelf_sv.
  - ``"tf32-refine"``: the row sketches in FP32 on the tcgen05 tensor cores (K split into
    two TF32 parts, ``opts["sketch"] = 1``) at the loose tolerance ``REFINE_FACTOR_TOL``,
    then FP64 iterative refinement against the on-the-fly FP64 matvec (stationary steps
    for symm 'n'/'s', preconditioned conjugate gradients for 'p') until every column's
    relative residual is below ``tol``.

Refinement adds at least two O(N^2 nrhs) FP64 products (the residuals) to a factorization
that is cheap because its tolerance is loose.  That pays in 3D, where the ranks -- and the
cost of a tight factorization -- grow quickly with 1/tol, as long as N nrhs keeps the
products short; on curves in 2D the ranks grow like log(1/tol) and the FP64-sketched
factorization at ``tol`` costs less than the two residual products.
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PREDICTOR_WEIGHTS = os.path.join(HERE, "predictor_weights.npz")
REFINE_FACTOR_TOL = 1e-6
REFINE_MAX_ITER = 10
# refinement only while N * nrhs stays at most this (two residual products of
# 2 N^2 nrhs flop each take well under a second on the FP64 tensor path)
REFINE_MAX_N_NRHS = 1 << 23
NOT_SPD = 2   # FLAM_ERR_NOT_SPD (FLAM:rskelf:notPosDef)


def choose(d, N, nrhs, tol, symm="n"):
    """The form :func:`solve` runs for a problem of N points in d dimensions with nrhs
    right-hand sides at target relative residual tol."""
    if tol >= REFINE_FACTOR_TOL:
        return "fp64-sketch"
    if d == 3 and symm != "p" and N * nrhs <= REFINE_MAX_N_NRHS:
        return "tf32-refine"
    return "fp64-sketch"


def load_predictor():
    """The trained rank predictor shipped with the package."""
    from .api import Predictor
    return Predictor.load(PREDICTOR_WEIGHTS)


def factor_opts(form, symm, predictor=None, stream=None, profile=False):
    """rskelf options of a form (the factorization tolerance is factor_tol(form, tol))."""
    o = dict(symm=symm, sketch=2 if form == "fp64-sketch" else 1, profile=profile)
    if predictor is not None:
        o.update(predictor=predictor, sketch_p=12)
    if stream is not None:
        o["stream"] = stream
    return o


def factor_tol(form, tol):
    return REFINE_FACTOR_TOL if form == "tf32-refine" else tol


def solve(A, x, occ, pxyfun, B, X, tol=1e-10, symm="n", predictor=None, form=None, stream=None, profile=False,
          max_iter=REFINE_MAX_ITER):
    """Factor A on points x in the chosen form and solve A X = B to relative residual tol.

    B and X are device tensors (N x nrhs, column-major); X is overwritten.  Returns
    (F, form, refinement steps, per-column relative residual or None).  With symm 'p', a
    sketched factorization that fails the positive-definite check of a redundant block is
    redone with symm 'n' (LU of the same matrix); ``F.symm`` tells which ran.  The residual is
    measured by the refinement itself in the "tf32-refine" form; the "fp64-sketch" form
    computes none (check it with ``F.matvec_``)."""
    d, N = int(x.shape[0]), int(x.shape[1])
    nrhs = int(B.shape[1]) if B.ndim == 2 else 1
    form = form or choose(d, N, nrhs, tol, symm)
    from ._lib import FlamError
    from .api import rskelf
    try:
        F = rskelf(A, x, occ, factor_tol(form, tol), pxyfun, factor_opts(form, symm, predictor, stream, profile))
    except FlamError as e:
        if symm != "p" or e.code != NOT_SPD:
            raise
        # The exact ID keeps every Schur complement of an SPD matrix SPD; a sketched ID's
        # interpolation error can leave a redundant block indefinite at the level of the
        # tolerance (seen on Matern covariances whose ranks fill the sketch).  The form
        # then factors the same symmetric matrix with LU (symm 'n').
        symm = "n"
        F = rskelf(A, x, occ, factor_tol(form, tol), pxyfun, factor_opts(form, symm, predictor, stream, profile))
    if form == "tf32-refine":
        _, it, rel = F.ir_sv_(B, X, tol, max_iter)
        return F, form, it, np.asarray(rel)
    X.copy_(B)
    F.sv_(X)
    return F, form, 0, None
