"""Recursive skeletonization factorization (oracle restatement).

``rskelf``      rskelf/rskelf.m:109-309
``rskelf_sv``   rskelf/rskelf_sv.m:13-36 and rskelf/sv/rskelf_sv_{nn,nc,sn,sc,h,p}.m
``rskelf_mv``   rskelf/rskelf_mv.m:13-36 and rskelf/mv/rskelf_mv_{nn,nc,sn,sc,h,p}.m

0-based indices throughout.  Real arithmetic only (the registry kernels are
real), so ``'t'`` and ``'c'`` coincide and ``'s'`` differs from ``'n'`` only in
the rows of the compressed block (rskelf.m:211) and ``T.'`` vs ``T'``.

``order="reference"`` processes the boxes of a level one after another, as
rskelf.m:184-261 does: a box sees same-level neighbours that were compressed
earlier in the loop as their skeletons only.  ``order="level_sync"`` gives
every box of a level the neighbour point sets as they stood after the
pull-up (rskelf.m:179-181), which is what a level-parallel device
implementation computes.
"""
import math
import time

import numpy as np
import scipy.linalg as sl

from .idecomp import id_
from .tree import hypoct


def chksymm(symm):
    """core/chksymm.m:8-13."""
    s = str(symm).lower()
    if s not in ("n", "s", "h", "p"):
        raise ValueError("FLAM:chksymm:invalidSymm: Symmetry parameter must be one of 'N', 'S', 'H', or 'P'.")
    return s


def chktrans(trans):
    """core/chktrans.m:8-13."""
    t = str(trans).lower()
    if t not in ("n", "t", "c"):
        raise ValueError("FLAM:chktrans:invalidTrans: Transpose parameter must be one of 'N', 'T', or 'C'.")
    return t


def _lu_vector(K):
    """MATLAB ``[L,U,p] = lu(K,'vector')`` (xGETRF): K[p] = L @ U."""
    n = K.shape[0]
    lu, piv = sl.lu_factor(K, check_finite=False)
    p = np.arange(n)
    for i, q in enumerate(piv):
        p[[i, q]] = p[[q, i]]
    L = np.tril(lu, -1) + np.eye(n)
    U = np.triu(lu)
    return L, U, p


def _rsolve_upper(B, U):
    """B / U for upper-triangular U."""
    if B.size == 0:
        return B.copy()
    return sl.solve_triangular(U, B.T, trans="T", lower=False, check_finite=False).T


def _rsolve_lower_t(B, L):
    """B / L' for lower-triangular L."""
    if B.size == 0:
        return B.copy()
    return sl.solve_triangular(L, B.T, lower=True, check_finite=False).T


def rskelf(A, x, occ, rank_or_tol, pxyfun=None, opts=None, order="reference", tree=None):
    """F = rskelf(A, x, occ, rank_or_tol, pxyfun, opts).  rskelf/rskelf.m:109-309."""
    opts = dict(opts or {})
    opts.setdefault("lvlmax", math.inf)
    opts.setdefault("ext", None)
    opts.setdefault("Tmax", 2.0)
    opts.setdefault("rrqr_iter", math.inf)
    opts.setdefault("symm", "n")
    opts.setdefault("stop", math.inf)
    opts.setdefault("verb", 0)
    symm = chksymm(opts["symm"])
    stop = opts["stop"]
    if stop is None:
        stop_fn = lambda lvl, l: False  # noqa: E731
    elif callable(stop):
        stop_fn = stop
    else:
        stop_fn = lambda lvl, l, s=stop: lvl >= s  # noqa: E731   rskelf.m:128
    x = np.asarray(x, dtype=np.float64)
    N = x.shape[1]
    ts = time.perf_counter()
    t = tree if tree is not None else hypoct(x, occ, opts["lvlmax"], opts["ext"])
    t_tree = time.perf_counter() - ts
    lvp = t["lvp"]
    nbox = int(lvp[-1])
    # count nonempty boxes at each level (rskelf.m:146-152)
    pblk = np.zeros(t["nlvl"] + 1, dtype=np.int64)
    for L in range(1, t["nlvl"] + 1):
        pblk[L] = pblk[L - 1] + sum(1 for i in range(lvp[L - 1], lvp[L]) if len(t["xi"][i]) > 0)
    xi = [a.copy() for a in t["xi"]]
    factors = []
    Flvp = [0]
    rem = np.ones(N, dtype=bool)
    M = [None] * nbox
    Mi = [None] * nbox
    P = np.zeros(N, dtype=np.int64)
    stats = []
    for lvl in range(t["nlvl"], 0, -1):
        l = t["l"][:, lvl - 1]
        if stop_fn(t["nlvl"] - lvl, l):                           # rskelf.m:172
            break
        ts = time.perf_counter()
        nrem1 = int(rem.sum())
        boxes = range(lvp[lvl - 1], lvp[lvl])
        for i in boxes:                                            # rskelf.m:179-181
            xi[i] = np.concatenate([xi[i]] + [xi[c] for c in t["chld"][i]]).astype(np.int64)
        snap = [a for a in xi] if order == "level_sync" else None
        # global compression (no pxyfun) sees the points remaining when the level starts in
        # the level-synchronous order, and rem as each box leaves it in the reference's
        rem_nbr = rem.copy() if order == "level_sync" else rem
        for i in boxes:
            slf = xi[i]
            src = snap if snap is not None else xi
            nb = t["nbor"][i]
            nbr = np.concatenate([src[j] for j in nb]).astype(np.int64) if len(nb) else np.zeros(0, np.int64)
            nslf = len(slf)
            Mbox = np.zeros((nslf, nslf))                          # rskelf.m:190-199
            if lvl < t["nlvl"]:
                P[slf] = np.arange(nslf)
                for j in t["chld"][i]:
                    k = P[xi[j]]
                    Mbox[np.ix_(k, k)] = M[j]
                    M[j] = None
                    Mi[j] = None
            M[i] = Mbox
            Mi[i] = slf
            Kpxy = np.zeros((0, nslf))
            if lvl > 2:                                            # rskelf.m:203-207
                if pxyfun is None:
                    nbr = np.setdiff1d(np.flatnonzero(rem_nbr), slf)
                else:
                    Kpxy, nbr = pxyfun(x, slf, nbr, l, t["ctr"][i])
            K = A(nbr, slf)                                        # rskelf.m:210-212
            if symm == "n":
                K = np.concatenate([K, A(slf, nbr).T], axis=0)
            K = np.concatenate([K, Kpxy], axis=0)
            sk, rd, T, _ = id_(K, rank_or_tol, opts["Tmax"], opts["rrqr_iter"])
            if len(rd) == 0:                                       # rskelf.m:216
                continue
            K = A(slf, slf) + M[i]                                 # rskelf.m:219-223
            K[rd, :] = K[rd, :] - T.T @ K[sk, :]
            K[:, rd] = K[:, rd] - K[:, sk] @ T
            Lf = Uf = pf = E = G = None
            if symm in ("n", "s"):                                 # rskelf.m:224-227
                Lf, Uf, pf = _lu_vector(K[np.ix_(rd, rd)])
                E = _rsolve_upper(K[np.ix_(sk, rd)], Uf)
                G = sl.solve_triangular(Lf, K[np.ix_(rd[pf], sk)], lower=True, unit_diagonal=True,
                                        check_finite=False) if len(sk) else np.zeros((len(rd), 0))
                X = E @ G
            elif symm == "h":                                      # rskelf.m:228-233
                lu, dd, perm = sl.ldl(K[np.ix_(rd, rd)], lower=True, hermitian=True, check_finite=False)
                Lf = lu[perm]
                Uf = dd
                rd = rd[perm]
                T = T[:, perm]
                E = _rsolve_lower_t(K[np.ix_(sk, rd)], Lf)
                E = np.linalg.solve(Uf.T, E.T).T if E.size else E
                X = E @ (Uf @ E.T)
            else:                                                  # rskelf.m:234-237
                Lf = np.linalg.cholesky(K[np.ix_(rd, rd)])
                E = _rsolve_lower_t(K[np.ix_(sk, rd)], Lf)
                X = E @ E.T
            M[i] = M[i][np.ix_(sk, sk)] - X                        # rskelf.m:245-246
            Mi[i] = slf[sk]
            factors.append(dict(sk=slf[sk].copy(), rd=slf[rd].copy(), T=T, L=Lf, U=Uf, p=pf, E=E, F=G))
            xi[i] = slf[sk].copy()                                 # rskelf.m:260-261
            rem[slf[rd]] = False
        Flvp.append(len(factors))
        te = time.perf_counter() - ts
        nblk = int(pblk[lvl - 1] + (lvp[lvl] - lvp[lvl - 1]))
        stats.append(dict(lvl=lvl, nblk=nblk, nrem1=nrem1, nrem2=int(rem.sum()), time=te))
    F = dict(N=N, nlvl=t["nlvl"], lvp=np.asarray(Flvp, dtype=np.int64), factors=factors, symm=symm,
             stats=stats, t_tree=t_tree, tree=t)
    Sn = int(rem.sum())
    if Sn:                                                         # rskelf.m:280-308
        Si = np.flatnonzero(rem)
        P[Si] = np.arange(Sn)
        S = np.zeros((Sn, Sn))
        for i in range(nbox):
            if M[i] is None or M[i].size == 0:
                continue
            idx = P[Mi[i]]
            S[np.ix_(idx, idx)] += M[i]
        F["Si"] = Si
        F["S"] = S
    return F


def _sv(F, X, trans):
    symm = F["symm"]
    fs = F["factors"]
    n = len(fs)
    sol = sl.solve_triangular
    if symm in ("n", "s") and trans == "n":                        # sv/rskelf_sv_nn.m, _sn.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["T"].T @ X[sk]
            X[rd] = sol(f["L"], X[rd[f["p"]]], lower=True, unit_diagonal=True)
            X[sk] -= f["E"] @ X[rd]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["F"] @ X[sk]
            X[rd] = sol(f["U"], X[rd], lower=False)
            X[sk] -= f["T"] @ X[rd]
    elif symm in ("n", "s"):                                       # sv/rskelf_sv_nc.m, _sc.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["T"].T @ X[sk]
            X[rd] = sol(f["U"], X[rd], trans="T", lower=False)
            X[sk] -= f["F"].T @ X[rd]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["E"].T @ X[sk]
            X[rd[f["p"]]] = sol(f["L"], X[rd], trans="T", lower=True, unit_diagonal=True)
            X[sk] -= f["T"] @ X[rd]
    elif symm == "h":                                              # sv/rskelf_sv_h.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["T"].T @ X[sk]
            X[rd] = sol(f["L"], X[rd], lower=True, unit_diagonal=True)
            X[sk] -= f["E"] @ X[rd]
            X[rd] = np.linalg.solve(f["U"], X[rd])
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["E"].T @ X[sk]
            X[rd] = sol(f["L"], X[rd], trans="T", lower=True, unit_diagonal=True)
            X[sk] -= f["T"] @ X[rd]
    else:                                                          # sv/rskelf_sv_p.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["T"].T @ X[sk]
            X[rd] = sol(f["L"], X[rd], lower=True)
            X[sk] -= f["E"] @ X[rd]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[rd] -= f["E"].T @ X[sk]
            X[rd] = sol(f["L"], X[rd], trans="T", lower=True)
            X[sk] -= f["T"] @ X[rd]
    del n
    return X


def _mv(F, X, trans):
    symm = F["symm"]
    fs = F["factors"]
    if symm in ("n", "s") and trans == "n":                        # mv/rskelf_mv_nn.m, _sn.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["T"] @ X[rd]
            X[rd] = f["U"] @ X[rd]
            X[rd] += f["F"] @ X[sk]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["E"] @ X[rd]
            X[rd[f["p"]]] = f["L"] @ X[rd]
            X[rd] += f["T"].T @ X[sk]
    elif symm in ("n", "s"):                                       # mv/rskelf_mv_nc.m, _sc.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["T"] @ X[rd]
            X[rd] = f["L"].T @ X[rd[f["p"]]]
            X[rd] += f["E"].T @ X[sk]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["F"].T @ X[rd]
            X[rd] = f["U"].T @ X[rd]
            X[rd] += f["T"].T @ X[sk]
    elif symm == "h":                                              # mv/rskelf_mv_h.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["T"] @ X[rd]
            X[rd] = f["L"].T @ X[rd]
            X[rd] += f["E"].T @ X[sk]
            X[rd] = f["U"] @ X[rd]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["E"] @ X[rd]
            X[rd] = f["L"] @ X[rd]
            X[rd] += f["T"].T @ X[sk]
    else:                                                          # mv/rskelf_mv_p.m
        for f in fs:
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["T"] @ X[rd]
            X[rd] = f["L"].T @ X[rd]
            X[rd] += f["E"].T @ X[sk]
        for f in reversed(fs):
            sk, rd = f["sk"], f["rd"]
            X[sk] += f["E"] @ X[rd]
            X[rd] = f["L"] @ X[rd]
            X[rd] += f["T"].T @ X[sk]
    return X


def rskelf_sv(F, X, trans="n"):
    """Y = rskelf_sv(F, X, trans).  rskelf/rskelf_sv.m:13-36 (X is N x nrhs)."""
    trans = chktrans(trans)
    X = np.array(X, dtype=np.float64, copy=True)
    vec = X.ndim == 1
    if vec:
        X = X[:, None]
    t = "n" if trans == "n" else "c"          # real data: 't' == 'c' (rskelf_sv.m:22)
    Y = _sv(F, X, t)
    return Y[:, 0] if vec else Y


def rskelf_mv(F, X, trans="n"):
    """Y = rskelf_mv(F, X, trans).  rskelf/rskelf_mv.m:13-36."""
    trans = chktrans(trans)
    X = np.array(X, dtype=np.float64, copy=True)
    vec = X.ndim == 1
    if vec:
        X = X[:, None]
    t = "n" if trans == "n" else "c"
    Y = _mv(F, X, t)
    return Y[:, 0] if vec else Y


def print_stats(F):
    """The ``opts.verb`` table of rskelf.m:131-136,267-272."""
    lines = ["-" * 69,
             "%3s | %6s | %19s | %19s | %10s" % ("lvl", "nblk", "start/end npts", "start/end npts/blk", "time (s)"),
             "-" * 69,
             "%3s | %63.2e" % ("t", F["t_tree"])]
    for s in F["stats"]:
        lines.append("%3d | %6d | %8d | %8d | %8.2f | %8.2f | %10.2e" % (
            s["lvl"], s["nblk"], s["nrem1"], s["nrem2"], s["nrem1"] / s["nblk"], s["nrem2"] / s["nblk"], s["time"]))
    lines.append("-" * 69)
    return "\n".join(lines)


def _sv_half(F, X, trans, upward):
    sol = sl.solve_triangular
    symm = F["symm"]
    fs = F["factors"] if upward else list(reversed(F["factors"]))
    for f in fs:
        sk, rd = f["sk"], f["rd"]
        if upward:
            X[rd] -= f["T"].T @ X[sk]
            if symm in ("n", "s") and trans == "n":
                X[rd] = sol(f["L"], X[rd[f["p"]]], lower=True, unit_diagonal=True)
                X[sk] -= f["E"] @ X[rd]
            elif symm in ("n", "s"):
                X[rd] = sol(f["U"], X[rd], trans="T", lower=False)
                X[sk] -= f["F"].T @ X[rd]
            elif symm == "h":
                X[rd] = sol(f["L"], X[rd], lower=True, unit_diagonal=True)
                X[sk] -= f["E"] @ X[rd]
                X[rd] = np.linalg.solve(f["U"], X[rd])
            else:
                X[rd] = sol(f["L"], X[rd], lower=True)
                X[sk] -= f["E"] @ X[rd]
        else:
            if symm in ("n", "s") and trans == "n":
                X[rd] -= f["F"] @ X[sk]
                X[rd] = sol(f["U"], X[rd], lower=False)
            elif symm in ("n", "s"):
                X[rd] -= f["E"].T @ X[sk]
                X[rd[f["p"]]] = sol(f["L"], X[rd], trans="T", lower=True, unit_diagonal=True)
            elif symm == "h":
                X[rd] -= f["E"].T @ X[sk]
                X[rd] = sol(f["L"], X[rd], trans="T", lower=True, unit_diagonal=True)
            else:
                X[rd] -= f["E"].T @ X[sk]
                X[rd] = sol(f["L"], X[rd], trans="T", lower=True)
            X[sk] -= f["T"] @ X[rd]
    return X


def _mv_half(F, X, trans, upward):
    symm = F["symm"]
    fs = F["factors"] if upward else list(reversed(F["factors"]))
    for f in fs:
        sk, rd = f["sk"], f["rd"]
        if upward:
            X[sk] += f["T"] @ X[rd]
            if symm in ("n", "s") and trans == "n":
                X[rd] = f["U"] @ X[rd]
                X[rd] += f["F"] @ X[sk]
            elif symm in ("n", "s"):
                X[rd] = f["L"].T @ X[rd[f["p"]]]
                X[rd] += f["E"].T @ X[sk]
            elif symm == "h":
                X[rd] = f["L"].T @ X[rd]
                X[rd] += f["E"].T @ X[sk]
                X[rd] = f["U"] @ X[rd]
            else:
                X[rd] = f["L"].T @ X[rd]
                X[rd] += f["E"].T @ X[sk]
        else:
            if symm in ("n", "s") and trans == "n":
                X[sk] += f["E"] @ X[rd]
                X[rd[f["p"]]] = f["L"] @ X[rd]
            elif symm in ("n", "s"):
                X[sk] += f["F"].T @ X[rd]
                X[rd] = f["U"].T @ X[rd]
            else:
                X[sk] += f["E"] @ X[rd]
                X[rd] = f["L"] @ X[rd]
            X[rd] += f["T"].T @ X[sk]
    return X


def _prep(X):
    X = np.array(X, dtype=np.float64, copy=True)
    vec = X.ndim == 1
    return (X[:, None] if vec else X), vec


def rskelf_cholmv(F, X, trans="n"):
    """Y = C X with F = C C' (symm 'p').  rskelf/rskelf_cholmv.m:15-50."""
    if F["symm"] != "p":
        raise ValueError("FLAM:rskelf_cholmv:invalidSymm: Symmetry parameter must be 'P'.")
    trans = chktrans(trans)
    X, vec = _prep(X)
    Y = _mv_half(F, X, "n", upward=(trans != "n"))     # 'n': downward half; 'c'/'t': upward half
    return Y[:, 0] if vec else Y


def rskelf_cholsv(F, X, trans="n"):
    """Y = C \\ X.  rskelf/rskelf_cholsv.m:15-50."""
    if F["symm"] != "p":
        raise ValueError("FLAM:rskelf_cholsv:invalidSymm: Symmetry parameter must be 'P'.")
    trans = chktrans(trans)
    X, vec = _prep(X)
    Y = _sv_half(F, X, "n", upward=(trans == "n"))     # 'n': upward half; 'c'/'t': downward half
    return Y[:, 0] if vec else Y


def rskelf_logdet(F):
    """log det of the factored matrix, imaginary part in [0, 2 pi).  rskelf/rskelf_logdet.m:11-33."""
    ld = 0.0 + 0.0j
    for f in F["factors"]:
        if F["symm"] == "p":
            ld += 2 * np.sum(np.log(np.diag(f["L"]).astype(complex)))
        elif F["symm"] == "h":
            ld += _logdet_ldl(f["U"])                                   # core/logdet_ldl.m
        else:
            ld += np.sum(np.log(np.diag(f["U"]).astype(complex))) + np.log(complex(_detperm(f["p"])))
    return complex(ld.real, math.fmod(ld.imag, 2 * math.pi) % (2 * math.pi))


def _detperm(p):
    """Sign of a permutation (compat/detperm.m)."""
    p = np.asarray(p)
    seen = np.zeros(len(p), dtype=bool)
    sgn = 1
    for i in range(len(p)):
        if not seen[i]:
            j, L = i, 0
            while not seen[j]:
                seen[j] = True
                j = p[j]
                L += 1
            if L % 2 == 0:
                sgn = -sgn
    return sgn


def _logdet_ldl(D):
    """core/logdet_ldl.m:6-12: 1x1 and 2x2 diagonal blocks of D."""
    D = np.asarray(D)
    one = np.count_nonzero(D, axis=0) == 1
    ld = np.sum(np.log(np.diag(D)[one].astype(complex)))
    idx = np.flatnonzero(~one)
    for i in range(0, len(idx), 2):
        b = D[np.ix_(idx[i:i + 2], idx[i:i + 2])]
        ld += np.log(complex(np.linalg.det(b)))
    return ld


def rskelf_partial_info(F):
    """[sk, S] = rskelf_partial_info(F).  rskelf/rskelf_partial_info.m."""
    if "Si" in F:
        return F["Si"], F["S"]
    return np.zeros(0, np.int64), np.zeros((0, 0))


def rskelf_partial_sv(F, X, svfun, trans="n"):
    """Upward sweep, svfun on X(Si), downward sweep.  rskelf/rskelf_partial_sv.m:23-62."""
    trans = chktrans(trans)
    X, vec = _prep(X)
    t = "n" if trans == "n" else "c"
    X = _sv_half(F, X, t, True)
    if "Si" in F and len(F["Si"]):
        X[F["Si"]] = svfun(X[F["Si"]], t)
    X = _sv_half(F, X, t, False)
    return X[:, 0] if vec else X


def rskelf_partial_mv(F, X, mvfun, trans="n"):
    """Upward sweep, mvfun on X(Si), downward sweep.  rskelf/rskelf_partial_mv.m."""
    trans = chktrans(trans)
    X, vec = _prep(X)
    t = "n" if trans == "n" else "c"
    X = _mv_half(F, X, t, True)
    if "Si" in F and len(F["Si"]):
        X[F["Si"]] = mvfun(X[F["Si"]], t)
    X = _mv_half(F, X, t, False)
    return X[:, 0] if vec else X


def rskelf_diag(F, dinv=0):
    """D = rskelf_diag(F, dinv): diag(F) (dinv 0) or diag(inv(F)) (dinv 1) by unfolding the
    factorization top-down on the sparse pattern of required entries.
    rskelf/rskelf_diag.m:35-185 (symm n, s, p)."""
    import scipy.sparse as sp
    N, symm = F["N"], F["symm"]
    lvp = np.asarray(F["lvp"])
    nlvl = len(lvp) - 1
    fs = F["factors"]
    rem = np.ones(N, dtype=bool)
    keep = [None] * max(nlvl, 1)
    keep[0] = sp.csr_matrix((np.ones(N, dtype=bool), (np.arange(N), np.arange(N))), shape=(N, N))
    for lvl in range(1, nlvl):                       # rskelf_diag.m:59-86
        for f in fs[lvp[lvl - 1]:lvp[lvl]]:
            rem[f["rd"]] = False
        I_, J_ = keep[lvl - 1].nonzero()
        m = rem[I_] & rem[J_]
        Is, Js = [I_[m]], [J_[m]]
        for f in fs[lvp[lvl - 1]:lvp[lvl]]:
            a, b = np.meshgrid(f["sk"], f["sk"], indexing="ij")
            Is.append(a.ravel())
            Js.append(b.ravel())
        I = np.concatenate(Is).astype(np.int64)
        J = np.concatenate(Js).astype(np.int64)
        if symm != "n":
            m = I >= J
            I, J = I[m], J[m]
        keep[lvl] = sp.csr_matrix((np.ones(len(I), dtype=bool), (I, J)), shape=(N, N))
        keep[lvl].sum_duplicates()
        keep[lvl].data[:] = True
    M = sp.csr_matrix((N, N))
    for lvl in range(nlvl, 0, -1):                   # rskelf_diag.m:97-177
        Ms = M.tocoo()
        Is, Js, Vs = [Ms.row], [Ms.col], [Ms.data]
        for f in fs[lvp[lvl - 1]:lvp[lvl]]:
            sk, rd = f["sk"], f["rd"]
            T, Lf, E = f["T"], f["L"], f["E"]
            if symm in ("n", "s"):
                U, G, p = f["U"], f["F"], f["p"]
            else:
                U, G, p = Lf.T, E.T, None
            nrd, nsk = len(rd), len(sk)
            ird = np.arange(nrd)
            isk = nrd + np.arange(nsk)
            X = np.zeros((nrd + nsk, nrd + nsk))
            X[np.ix_(ird, ird)] = np.eye(nrd)
            Xsk = M[sk][:, sk].toarray()
            if symm != "n":                          # spsymm (core/spsymm.m): one of each pair stored
                Xsk = Xsk + Xsk.T - np.diag(np.diag(Xsk))
            X[np.ix_(isk, isk)] = Xsk
            if dinv:
                B = X[:, ird] - X[:, isk] @ E
                X[:, ird] = sl.solve_triangular(Lf, B.T, trans="T", lower=True,
                                                unit_diagonal=symm != "p").T
                X[ird, :] = sl.solve_triangular(U, X[ird, :] - G @ X[isk, :], lower=False)
                if p is not None:
                    Xc = X[:, ird].copy()
                    X[:, ird[p]] = Xc
                X[:, isk] = X[:, isk] - X[:, ird] @ T.T
                X[isk, :] = X[isk, :] - T @ X[ird, :]
            else:
                X[:, isk] = X[:, isk] + X[:, ird] @ G
                X[isk, :] = X[isk, :] + E @ X[ird, :]
                X[:, ird] = X[:, ird] @ U
                X[ird, :] = Lf @ X[ird, :]
                if p is not None:
                    Xr = X[ird, :].copy()
                    X[ird[p], :] = Xr
                X[:, ird] = X[:, ird] + X[:, isk] @ T
                X[ird, :] = X[ird, :] + T.T @ X[isk, :]
            X[np.ix_(isk, isk)] -= Xsk
            idx = np.concatenate([rd, sk])
            a, b = np.meshgrid(idx, idx, indexing="ij")
            Is.append(a.ravel())
            Js.append(b.ravel())
            Vs.append(X.ravel())
        M = sp.csr_matrix((np.concatenate(Vs), (np.concatenate(Is), np.concatenate(Js))), shape=(N, N))
        M = M.multiply(keep[lvl - 1]).tocsr()
    return np.asarray(M.diagonal()).copy()
