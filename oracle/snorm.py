"""Randomized power-method spectral norm (oracle restatement of ``core/snorm.m:31-72``)."""
import warnings

import numpy as np


def snorm(n, mv, mva=None, tol=1e-2, herm=False, niter_max=32, rng=None):
    if tol is None:
        tol = 1e-2
    if not tol >= 0:
        raise ValueError("FLAM:snorm:invalidTol: Tolerance must be nonnegative.")
    if not niter_max > 0:
        raise ValueError("FLAM:snorm:invalidMaxIter: Maximum number of iterations must be positive.")
    rng = rng or np.random.default_rng(0)
    x = rng.random(n)
    xnorm = np.linalg.norm(x)
    s = xnorm
    for _ in range(niter_max):
        x = x / xnorm
        s_ = s
        x = mv(x) if herm else mva(mv(x))
        xnorm = np.linalg.norm(x)
        s = xnorm if herm else np.sqrt(xnorm)
        if xnorm <= np.finfo(float).eps:
            return s
        if abs(s - s_) <= s_ * tol:
            return s
    warnings.warn("FLAM:snorm:maxIterCount: Maximum number of iterations reached.")
    return s
