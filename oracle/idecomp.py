"""Interpolative decomposition (oracle restatement of ``core/id.m``).

0-based indices.  ``id_(A, rank_or_tol, Tmax, rrqr_iter)`` returns
``(sk, rd, T, niter)`` with ``A[:, rd] ~= A[:, sk] @ T``.

LAPACK routines the reference reaches through MATLAB built-ins are called
through SciPy: ``qr(A,0)`` with three outputs is xGEQP3 (``scipy.linalg.qr``
with ``pivoting=True``), the unpivoted row reduction is xGEQRF, the
triangular ``\\`` is xTRTRS.  ``qrupdate`` (used only to re-triangularise R11
after swapping two of its columns, id.m:134,217) is restated with Givens
rotations: the spike the swap leaves in column i is cleared bottom-up, then the
subdiagonal it leaves behind top-down (qrupdate's own rotation signs are not
pinned by any reference test).  In the tolerance mode every quantity the loop
reads from R11 (inverse row norms, ``R11\\r`` products, T) is invariant under
the row signs of R; the fixed-rank branch (id.m:168-198) is not, because it
sets ``R(k+1,k+1) = sqrt(c2(1))`` whatever sign the reflection produced.
"""
import math
import warnings

import numpy as np
import scipy.linalg as sl


def _tri_solve(R, b):
    if R.shape[0] == 0:
        return np.zeros_like(b)
    return sl.solve_triangular(R, b, lower=False, check_finite=False)


def _rot(a, b):
    if b == 0.0:
        return 1.0, 0.0
    r = math.hypot(a, b)
    return a / r, b / r


def _swap_r11(R, i, k):
    """Swap columns i and k-1 of R[:k,:k] and re-triangularise (id.m:134,217)."""
    R[:k, [i, k - 1]] = R[:k, [k - 1, i]]
    for row in range(k - 1, i, -1):              # spike in column i, bottom-up
        c, s = _rot(R[row - 1, i], R[row, i])
        a, b = R[row - 1, i:k].copy(), R[row, i:k].copy()
        R[row - 1, i:k] = c * a + s * b
        R[row, i:k] = -s * a + c * b
        R[row, i] = 0.0
    for col in range(i + 1, k - 1):              # subdiagonal left behind, top-down
        c, s = _rot(R[col, col], R[col + 1, col])
        a, b = R[col, col:k].copy(), R[col + 1, col:k].copy()
        R[col, col:k] = c * a + s * b
        R[col + 1, col:k] = -s * a + c * b
        R[col + 1, col] = 0.0


def id_(A, rank_or_tol, Tmax=2.0, rrqr_iter=math.inf):
    """core/id.m:44-248 (the ``fixed`` argument is not on the rskelf path)."""
    st = _id_qr(A, rank_or_tol, Tmax, rrqr_iter)
    if st[0] == "done":
        return st[1]
    _, R, p, k, tol, n = st
    return _id_rrqr(R, p, k, tol, n, Tmax, rrqr_iter)


def _id_qr(A, rank_or_tol, Tmax=2.0, rrqr_iter=math.inf):
    """id.m:44-114: argument checks, pivoted QR, rank, T stored in R."""
    if Tmax is None:
        Tmax = 2.0
    if rrqr_iter is None:
        rrqr_iter = math.inf
    if not rank_or_tol >= 0:
        raise ValueError("FLAM:id:invalidRankOrTol: Rank or tolerance must be nonnegative.")
    if not Tmax >= 1:
        raise ValueError("FLAM:id:invalidTmax: Interpolation matrix entry bound must be >= 1.")
    if not rrqr_iter >= 0:
        raise ValueError("FLAM:id:invalidRRQRIter: Maximum number of RRQR iterations must be nonnegative.")
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    niter = 0
    if m == 0 or n == 0:                                   # id.m:64-68
        return ("done", (np.zeros(0, np.int64), np.arange(n, dtype=np.int64), np.zeros((0, n)), 0))
    tol = math.fmod(rank_or_tol, 1.0)                      # id.m:71
    kmax = int(math.floor(rank_or_tol))                    # id.m:72
    if kmax == 0 or kmax > n:
        kmax = n
    if m > 8 * n:                                          # id.m:102
        A = sl.qr(A, mode="economic", check_finite=False)[1]
    _, R, p = sl.qr(A, mode="economic", pivoting=True, check_finite=False)   # id.m:105
    p = p.astype(np.int64)
    R = np.array(R)
    cmax = abs(R[0, 0])                                    # id.m:106
    tol = cmax * tol                                       # id.m:107
    if min(R.shape) == 1 or R.shape[0] == 1 or R.shape[1] == 1:
        diagR = np.array([R[0, 0]])                        # id.m:108
    else:
        diagR = np.diag(R)
    k = int(np.count_nonzero(np.abs(diagR) > tol))         # id.m:111
    R = R[:k, :].copy()                                    # id.m:112
    k = min(k, kmax)                                       # id.m:113
    if k > 0 and k < n:
        R[:k, k:] = _tri_solve(R[:k, :k], R[:k, k:])       # id.m:114
    return ("rrqr", R, p, k, tol, n)


def _id_rrqr(R, p, k, tol, n, Tmax, rrqr_iter):
    """id.m:116-240: RRQR refinement of (R with T stored, p, k) and the outputs."""
    if Tmax is None:
        Tmax = 2.0
    if rrqr_iter is None:
        rrqr_iter = math.inf
    niter = 0
    # RRQR refinement (id.m:117-236)
    if not math.isinf(Tmax) and rrqr_iter > 0 and 0 < k < n:
        f2 = Tmax ** 2
        c2 = np.sum(R[k:, k:] ** 2, axis=0) if R.shape[0] > k else np.zeros(n - k)
        r2 = np.sum(_tri_solve(R[:k, :k], np.eye(k)) ** 2, axis=1)
        conv = False
        while niter < rrqr_iter:
            tmp = R[:k, k:] ** 2 + np.outer(r2, c2)
            flat = np.abs(tmp).ravel(order="F")
            idx = int(np.argmax(flat))
            t2 = flat[idx]
            if t2 <= f2:
                conv = True
                break
            niter += 1
            i, j = idx % k, idx // k                       # id.m:129
            if i < k - 1:                                  # id.m:132-138
                p[[i, k - 1]] = p[[k - 1, i]]
                _swap_r11(R, i, k)
                R[[i, k - 1], k:] = R[[k - 1, i], k:]
                r2[[i, k - 1]] = r2[[k - 1, i]]
            if j > 0:                                      # id.m:141-145
                p[[k, k + j]] = p[[k + j, k]]
                R[:, [k, k + j]] = R[:, [k + j, k]]
                c2[[0, j]] = c2[[j, 0]]
            # downdate inverse row norms (id.m:148-149)
            r2[:k - 1] = r2[:k - 1] - np.abs(_tri_solve(R[:k - 1, :k - 1], R[:k - 1, k - 1]) / R[k - 1, k - 1]) ** 2
            r2[k - 1] = 0.0
            if R.shape[0] == k:                            # id.m:164-167
                u = R[:, k].copy()
                R[:, k] = R[:, :k] @ R[:, k]
                R[:k - 1, k - 1] = 0.0
                R[k - 1, k - 1] = 1.0
            else:                                          # id.m:168-198
                v = R[k:, k].copy()
                v[0] = v[0] + math.sqrt(c2[0]) * np.sign(R[k, k]) if R[k, k] != 0 else v[0] + math.sqrt(c2[0])
                v = v / np.linalg.norm(v)
                R[k:, k + 1:] = R[k:, k + 1:] - 2.0 * np.outer(v, v @ R[k:, k + 1:])
                R[k + 1:, k] = 0.0
                R[k, k] = math.sqrt(c2[0])
                R[:k, k] = R[:k, :k] @ R[:k, k]
                R[k - 1, k + 1:] = R[k - 1, k - 1] * R[k - 1, k + 1:]
                r = R[:k, k - 1].copy()
                s = R[k - 1, k + 1:].copy()
                c2 = c2 - np.abs(R[k, k:]) ** 2
                a_, b_ = R[k - 1, k], R[k, k]
                G = _givens(a_, b_)
                R[k - 1:k + 1, k - 1:] = G @ R[k - 1:k + 1, k - 1:]
                c2 = c2 + np.abs(R[k, k:]) ** 2
                c2[0] = abs(R[k, k - 1]) ** 2
                tmp_ = R[k - 1, k - 1]
                R[k - 1, k - 1] = r[k - 1]
                u = _tri_solve(R[:k, :k], R[:k, k])
                R[k - 1, k - 1] = tmp_
                vv = _tri_solve(R[:k - 1, :k - 1], r[:k - 1])
                R[k - 1, k - 1] = R[k - 1, k - 1] / r[k - 1]
                R[:k - 1, k - 1] = vv * (1.0 - R[k - 1, k - 1])
                R[:k - 1, k + 1:] = R[:k - 1, k + 1:] + np.outer(vv / r[k - 1], s - R[k - 1, k + 1:])
                R[k - 1, k + 1:] = R[k - 1, k + 1:] / r[k - 1]
            # swap k-th and (k+1)-th columns (id.m:201-204)
            p[[k - 1, k]] = p[[k, k - 1]]
            R[:, [k - 1, k]] = R[:, [k, k - 1]]
            r2[:k - 1] = r2[:k - 1] + np.abs(_tri_solve(R[:k - 1, :k - 1], R[:k - 1, k - 1]) / R[k - 1, k - 1]) ** 2
            r2[k - 1] = 1.0 / abs(R[k - 1, k - 1]) ** 2
            # Sherman-Morrison (id.m:207-208)
            u[k - 1] = u[k - 1] - 1.0
            R[:k, k:] = R[:k, k:] - np.outer(u, R[k - 1, k:]) / (1.0 + u[k - 1])
            # rank reduction (id.m:211-229)
            rr = 1.0 / np.sqrt(r2)
            i = int(np.argmin(rr))
            if rr[i] > tol:
                continue
            if i < k - 1:
                p[[i, k - 1]] = p[[k - 1, i]]
                _swap_r11(R, i, k)
                R[[i, k - 1], k:] = R[[k - 1, i], k:]
                r2[[i, k - 1]] = r2[[k - 1, i]]
            c2 = np.zeros(n - k + 1)
            r2 = r2[:k - 1] - np.abs(_tri_solve(R[:k - 1, :k - 1], R[:k - 1, k - 1]) / R[k - 1, k - 1]) ** 2
            k -= 1
            r = _tri_solve(R[:k, :k], R[:k, k])
            R[:k, k:] = np.concatenate([r[:, None], R[:k, k + 1:] + np.outer(r, R[k, k + 1:])], axis=1)
            R = R[:k, :].copy()
            if k == 0:
                break
        if not conv and k > 0:
            warnings.warn("FLAM:id:maxIterCount: Maximum number of RRQR iterations reached.")
    sk = p[:k].copy()
    rd = p[k:].copy()
    T = R[:k, k:].copy()
    return sk, rd, T, niter


def _givens(a, b):
    """MATLAB ``givens(a,b)`` for real input: G @ [a; b] = [sign(a) r; 0], c >= 0."""
    if a == 0:
        return np.array([[0.0, 1.0], [-1.0, 0.0]])
    r = math.hypot(a, b)
    c = abs(a) / r
    s = math.copysign(1.0, a) * (b / r)
    return np.array([[c, s], [-s, c]])
