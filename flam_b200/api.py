"""MATLAB-signature host API over the C ABI.

    F = rskelf(A, x, occ, rank_or_tol, pxyfun=None, opts=None)     rskelf/rskelf.m:109
    Y = rskelf_sv(F, X, trans='n')                                  rskelf/rskelf_sv.m:13
    Y = rskelf_mv(F, X, trans='n')                                  rskelf/rskelf_mv.m:13
    Y = rskelf_cholmv(F, X, trans='n')                              rskelf/rskelf_cholmv.m:15
    Y = rskelf_cholsv(F, X, trans='n')                              rskelf/rskelf_cholsv.m:15
    ld = rskelf_logdet(F)                                           rskelf/rskelf_logdet.m:11
    Si, S = rskelf_partial_info(F)                                  rskelf/rskelf_partial_info.m:12
    Y = rskelf_partial_sv(F, X, svfun, trans='n')                   rskelf/rskelf_partial_sv.m:23
    Y = rskelf_partial_mv(F, X, mvfun, trans='n')                   rskelf/rskelf_partial_mv.m:23
    T = hypoct(x, occ, lvlmax=inf, ext=None)                        core/hypoct.m:51
    P = hypoct_perm(T)                                              core/hypoct_perm.m:11

``A`` and ``pxyfun`` are registry descriptors (:class:`flam_b200.Kernel`,
:class:`flam_b200.Proxy`); a Python callable is rejected with
``FLAM:gpu:unsupportedHandle`` because the matrix is evaluated on the device.
Indices are 0-based.  ``X`` may be a NumPy array (host; copied in and out by
the library) or a CUDA tensor (device pointer, no host copies).
"""
import ctypes as C
import math

import numpy as np

from . import _lib
from .registry import Kernel, Proxy

_OPT_KEYS = {"lvlmax", "ext", "Tmax", "rrqr_iter", "symm", "stop", "verb", "stream", "profile", "sketch", "sketch_p",
             "sketch_guard", "sketch_seed", "predictor", "rank_log"}


def _c_opts(opts):
    o = _lib.FlamOpts()
    _lib.lib().flam_opts_default(C.byref(o))
    keep = []
    for k, v in (opts or {}).items():
        if k not in _OPT_KEYS:
            continue
        if k == "lvlmax":
            o.lvlmax = 0 if (v is None or v == math.inf) else int(v)
        elif k == "ext":
            if v is not None and np.size(v):
                e = np.asfortranarray(v, dtype=np.float64)
                keep.append(e)
                o.ext = e.ctypes.data
        elif k == "Tmax":
            o.Tmax = float(v)
        elif k == "rrqr_iter":
            o.rrqr_iter = -1 if (v is None or v == math.inf) else int(v)
        elif k == "symm":
            o.symm = str(v).encode()[:1]
        elif k == "stop":
            o.stop = -1 if (v is None or v == math.inf) else int(v)
        elif k == "verb":
            o.verb = int(bool(v))
        elif k == "stream":
            o.stream = v
        elif k == "profile":
            o.profile = int(bool(v))
        elif k in ("sketch", "sketch_p", "sketch_guard"):
            setattr(o, k, int(v))
        elif k == "sketch_seed":
            o.sketch_seed = int(v) & 0xFFFFFFFF
        elif k == "predictor":
            o.predictor = None if v is None else (v.handle if hasattr(v, "handle") else v)
        elif k == "rank_log":
            o.rank_log = int(bool(v))
    return o, keep


def _is_cuda_tensor(X):
    return type(X).__module__.startswith("torch") and getattr(X, "is_cuda", False)


class Factor:
    """Handle of a device factorization (the reference's struct ``F``)."""

    def __init__(self, handle, ninst=1, keep=None):
        self._h = handle
        self.ninst = ninst
        self._keep = keep
        self._free = _lib.lib().flam_factor_free

    def free(self):
        """Release the device memory now (the reference's ``clear F``)."""
        h = getattr(self, "_h", None)
        if h:
            self._free(h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self):
        i = _lib.FlamInfo()
        _lib.check(_lib.lib().flam_factor_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in i._fields_}

    @property
    def N(self):
        return self.info()["N"]

    @property
    def symm(self):
        return self.info()["symm"].decode()

    # ---------------------------------------------------------------- exports
    def tree(self, inst=0):
        """The reference's hypoct struct (0-based), see core/hypoct.m:15-37."""
        L = _lib.lib()
        i64 = C.c_int64
        nlvl, nbox, nc, nn, npt = C.c_int(), i64(), i64(), i64(), i64()
        _lib.check(L.flam_tree_export(self._h, inst, C.byref(nlvl), C.byref(nbox), C.byref(nc), C.byref(nn),
                                      C.byref(npt), *([None] * 11)))
        d = self.info()["d"]
        nb = nbox.value
        lvp = np.zeros(nlvl.value + 1, np.int64)
        lv = np.zeros(d * nlvl.value)
        ctr = np.zeros(d * nb)
        prnt = np.zeros(nb, np.int64)
        cp = np.zeros(nb + 1, np.int64)
        ch = np.zeros(max(nc.value, 1), np.int64)
        npp = np.zeros(nb + 1, np.int64)
        nbr = np.zeros(max(nn.value, 1), np.int64)
        xp = np.zeros(nb + 1, np.int64)
        xi = np.zeros(max(npt.value, 1), np.int64)
        p64 = lambda a: a.ctypes.data_as(C.POINTER(i64))  # noqa: E731
        pd = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        _lib.check(L.flam_tree_export(self._h, inst, C.byref(nlvl), C.byref(nbox), C.byref(nc), C.byref(nn),
                                      C.byref(npt), p64(lvp), pd(lv), pd(ctr), p64(prnt), p64(cp), p64(ch),
                                      p64(npp), p64(nbr), p64(xp), p64(xi)))
        return dict(nlvl=nlvl.value, lvp=lvp, l=lv.reshape(nlvl.value, d).T.copy(), ctr=ctr.reshape(nb, d),
                    prnt=prnt, chld=[ch[cp[b]:cp[b + 1]] for b in range(nb)],
                    nbor=[nbr[npp[b]:npp[b + 1]] for b in range(nb)], xi=[xi[xp[b]:xp[b + 1]] for b in range(nb)])

    def perm(self, inst=0):
        n = int(self._inst_sizes()[inst])
        P = np.zeros(n, np.int64)
        _lib.check(_lib.lib().flam_tree_perm(self._h, inst, P.ctypes.data_as(C.POINTER(C.c_int64))))
        return P

    def _inst_sizes(self):
        sizes = getattr(self, "_sizes", None)
        if sizes is None:
            sizes = [sum(len(a) for a in self.tree(i)["xi"]) for i in range(self.ninst)]
            self._sizes = sizes
        return sizes

    def factors(self, inst=0):
        """The reference's ``F`` struct: lvp, factors(i).{sk,rd,T,L,U,p,E,F} (rskelf.m:157-159,249-257)."""
        L = _lib.lib()
        i64 = C.c_int64
        nfac, nlvp = i64(), C.c_int()
        _lib.check(L.flam_factor_sizes(self._h, inst, C.byref(nfac), C.byref(nlvp), None, None, None))
        lvp = np.zeros(nlvp.value, np.int64)
        k = np.zeros(max(nfac.value, 1), np.int64)
        r = np.zeros(max(nfac.value, 1), np.int64)
        p64 = lambda a: a.ctypes.data_as(C.POINTER(i64))  # noqa: E731
        pd = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
        _lib.check(L.flam_factor_sizes(self._h, inst, C.byref(nfac), C.byref(nlvp), p64(lvp), p64(k), p64(r)))
        symm = self.symm
        out = []
        for j in range(nfac.value):
            kk, rr = int(k[j]), int(r[j])
            sk = np.zeros(max(kk, 1), np.int64)
            rd = np.zeros(max(rr, 1), np.int64)
            T = np.zeros((kk, rr), order="F")
            Lm = np.zeros((rr, rr), order="F")
            U = np.zeros((rr, rr), order="F")
            p = np.zeros(max(rr, 1), np.int64)
            E = np.zeros((kk, rr), order="F")
            G = np.zeros((rr, kk), order="F")
            _lib.check(L.flam_factor_export(self._h, inst, j, p64(sk), p64(rd), pd(T), pd(Lm), pd(U), p64(p),
                                            pd(E), pd(G)))
            f = dict(sk=sk[:kk], rd=rd[:rr], T=np.ascontiguousarray(T), L=np.ascontiguousarray(Lm), E=np.ascontiguousarray(E))
            if symm == "p":
                f.update(U=None, p=None, F=None)
            else:
                f.update(U=np.ascontiguousarray(U), p=p[:rr], F=np.ascontiguousarray(G))
            out.append(f)
        return dict(N=self._inst_sizes()[inst], lvp=lvp, factors=out, symm=symm)

    def profile(self, reset=False):
        """Launch accounting (kernel times, algorithmic flops/bytes, launch counts)."""
        p = _lib.FlamProf()
        _lib.check(_lib.lib().flam_profile(self._h, C.byref(p), int(bool(reset))))
        return {f: getattr(p, f) for f, _ in p._fields_}

    def level_stats(self, inst=0):
        """Rows (lvl, nblk, start npts, end npts) of the opts.verb table (rskelf.m:267-272)."""
        n = C.c_int()
        _lib.check(_lib.lib().flam_level_stats(self._h, inst, C.byref(n), None))
        rows = np.zeros(4 * max(n.value, 1), np.int64)
        _lib.check(_lib.lib().flam_level_stats(self._h, inst, C.byref(n), rows.ctypes.data_as(C.POINTER(C.c_int64))))
        return rows[:4 * n.value].reshape(n.value, 4)

    # ---------------------------------------------------------------- apply
    def sv_(self, X, trans="n"):
        """In-place solve on a CUDA tensor or Fortran-ordered float64 NumPy array."""
        return self._apply(X, trans, True)

    def mv_(self, X, trans="n"):
        return self._apply(X, trans, False)

    def _apply(self, X, trans, solve, name=None, extra=()):
        L = _lib.lib()
        fn = getattr(L, name) if name else (L.flam_rskelf_sv if solve else L.flam_rskelf_mv)
        if _is_cuda_tensor(X):
            import torch
            if X.dtype != torch.float64:
                raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: X must be float64")
            if X.dim() == 1:
                ptr, ld, nrhs = X.data_ptr(), X.shape[0], 1
            else:
                if X.stride(0) != 1:
                    raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: X must be column-major (X.t().contiguous().t())")
                ptr, ld, nrhs = X.data_ptr(), X.stride(1), X.shape[1]
            _lib.check(fn(self._h, C.c_void_p(ptr), ld, nrhs, str(trans).encode()[:1], *extra))
            return X
        if not (isinstance(X, np.ndarray) and X.dtype == np.float64 and (X.ndim == 1 or X.flags.f_contiguous)):
            raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: X must be a float64 Fortran-ordered array")
        nrhs = 1 if X.ndim == 1 else X.shape[1]
        _lib.check(fn(self._h, C.c_void_p(X.ctypes.data), X.shape[0], nrhs, str(trans).encode()[:1], *extra))
        return X

    # ------------------------------------------------------- FP64 products and refinement
    @staticmethod
    def _block(X, name):
        """(pointer, leading dimension, columns) of a float64 column-major CUDA tensor or NumPy array."""
        if _is_cuda_tensor(X):
            import torch
            if X.dtype != torch.float64:
                raise _lib.FlamError(1, f"FLAM:{name}:invalidArg: arrays must be float64")
            if X.dim() == 1:
                return X.data_ptr(), X.shape[0], 1
            if X.stride(0) != 1:
                raise _lib.FlamError(1, f"FLAM:{name}:invalidArg: arrays must be column-major")
            return X.data_ptr(), X.stride(1), X.shape[1]
        if not (isinstance(X, np.ndarray) and X.dtype == np.float64 and (X.ndim == 1 or X.flags.f_contiguous)):
            raise _lib.FlamError(1, f"FLAM:{name}:invalidArg: arrays must be float64 Fortran-ordered")
        return X.ctypes.data, X.shape[0], 1 if X.ndim == 1 else X.shape[1]

    def matvec_(self, X, Y, B=None):
        """Y = A X (or B - A X) with the handle's registry matrix in FP64 (flam_matvec)."""
        px, lx, nrhs = self._block(X, "matvec")
        py, ly, ny = self._block(Y, "matvec")
        pb, lb = (None, 1) if B is None else self._block(B, "matvec")[:2]
        if ny != nrhs:
            raise _lib.FlamError(1, "FLAM:matvec:invalidArg: X and Y need the same number of columns")
        _lib.check(_lib.lib().flam_matvec(self._h, C.c_void_p(px), lx, nrhs, None if pb is None else C.c_void_p(pb),
                                          lb, C.c_void_p(py), ly))
        return Y

    def ir_sv_(self, B, X, ir_tol=1e-10, max_iter=10):
        """X = A \\ B by FP64 iterative refinement on this factorization (flam_rskelf_ir_sv).
        Returns (X, refinement steps, per-column FP64 relative residuals)."""
        pb, lb, nrhs = self._block(B, "rskelf_ir_sv")
        px, lx, nx = self._block(X, "rskelf_ir_sv")
        if nx != nrhs:
            raise _lib.FlamError(1, "FLAM:rskelf_ir_sv:invalidArg: B and X need the same number of columns")
        it = C.c_int()
        rel = np.zeros(max(nrhs, 1))
        _lib.check(_lib.lib().flam_rskelf_ir_sv(self._h, C.c_void_p(pb), lb, C.c_void_p(px), lx, nrhs, float(ir_tol),
                                                int(max_iter), C.byref(it),
                                                rel.ctypes.data_as(C.POINTER(C.c_double))))
        return X, it.value, rel[:nrhs]

    def rank_log(self):
        """(features, k/n) of every compressed box of a factorization made with opts rank_log."""
        L = _lib.lib()
        cnt = C.c_int64()
        _lib.check(L.flam_rank_log(self._h, C.byref(cnt), None, None))
        X = np.zeros((max(cnt.value, 1), 16), np.float32)
        y = np.zeros(max(cnt.value, 1), np.float32)
        fp = C.POINTER(C.c_float)
        _lib.check(L.flam_rank_log(self._h, C.byref(cnt), X.ctypes.data_as(fp), y.ctypes.data_as(fp)))
        return X[:cnt.value], y[:cnt.value]

    # ------------------------------------------------------- partial factorization
    def partial_info(self, inst=0):
        """[Si, S] = rskelf_partial_info(F): remaining skeletons (0-based, ascending) and the
        sparse update S, so that A(Si,Si) + S is the skeleton system left to the caller."""
        import scipy.sparse as sp
        L = _lib.lib()
        i64 = C.c_int64
        Sn, nnz = i64(), i64()
        _lib.check(L.flam_partial_sizes(self._h, inst, C.byref(Sn), C.byref(nnz)))
        n, z = Sn.value, nnz.value
        Si = np.zeros(max(n, 1), np.int64)
        cp = np.zeros(n + 1, np.int64)
        ri = np.zeros(max(z, 1), np.int64)
        v = np.zeros(max(z, 1))
        p64 = lambda a: a.ctypes.data_as(C.POINTER(i64))  # noqa: E731
        _lib.check(L.flam_partial_export(self._h, inst, p64(Si), p64(cp), p64(ri),
                                         v.ctypes.data_as(C.POINTER(C.c_double))))
        return Si[:n], sp.csc_matrix((v[:z], ri[:z], cp), shape=(n, n))

    def _partial(self, X, fun, trans, solve):
        host = not _is_cuda_tensor(X)
        err = []

        def cb(yptr, n, nrhs, tr, stream, ctx):
            try:
                import torch
                torch.cuda.synchronize()
                Y = torch.as_tensor(_DevBlock(yptr, n, nrhs), device="cuda")
                arg = Y.cpu().numpy().copy(order="F") if host else Y.clone()
                out = fun(arg, tr.decode())
                if tuple(np.shape(out)) != (n, nrhs) and not (nrhs == 1 and np.size(out) == n):
                    raise ValueError(f"skeleton function returned shape {np.shape(out)}, expected {(n, nrhs)}")
                Y.copy_(torch.as_tensor(np.asarray(out) if host else out, dtype=torch.float64).reshape(n, nrhs))
                torch.cuda.synchronize()
                return 0
            except Exception as e:  # noqa: BLE001 - re-raised after the call returns
                err.append(e)
                return 1

        cfn = _lib.SKEL_FN(cb)
        name = "flam_rskelf_partial_sv" if solve else "flam_rskelf_partial_mv"
        try:
            self._apply(X, trans, solve, name, (cfn, None))
        except _lib.FlamError:
            if err:
                raise err[0]
            raise
        return X



def _check_handles(A, pxyfun):
    if callable(A) and not isinstance(A, Kernel):
        raise _lib.FlamError(5, "FLAM:gpu:unsupportedHandle: A must be a registry Kernel, not a function handle")
    if pxyfun is not None and not isinstance(pxyfun, Proxy):
        raise _lib.FlamError(5, "FLAM:gpu:unsupportedHandle: pxyfun must be a registry Proxy, not a function handle")


def _points(x):
    """(pointer, d, N, keepalive) of d x N points: NumPy (host) or a CUDA tensor (device)."""
    if _is_cuda_tensor(x):
        import torch
        if x.dtype != torch.float64 or x.dim() != 2 or x.stride(0) != 1 or x.stride(1) != x.shape[0]:
            raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: x must be a float64 d x N column-major tensor "
                                    "(e.g. pts.t() of a contiguous N x d tensor)")
        return x.data_ptr(), x.shape[0], x.shape[1], x
    a = np.asfortranarray(x, dtype=np.float64)
    return a.ctypes.data, a.shape[0], a.shape[1], a


def _stop_levels(stop, x, occ, opts):
    """Levels an ``opts.stop`` predicate lets the factorization run (rskelf.m:128,172).

    The reference calls ``stop(nlvl - lvl, l)`` before each level (``l`` the level's box
    size, d values) and stops at the first true.  The levels and their sizes come from the
    tree alone, so the predicate is evaluated here on the tree rskelf builds (same occ,
    lvlmax and ext) and the library gets the equivalent level count."""
    if _is_cuda_tensor(x):
        x = x.detach().cpu().numpy()
    T = hypoct(x, occ, (opts or {}).get("lvlmax", math.inf), (opts or {}).get("ext"))
    try:
        t = T.tree()
    finally:
        T.free()
    nlvl, l = t["nlvl"], np.asarray(t["l"])
    for done in range(nlvl):
        if stop(done, l[:, nlvl - done - 1].copy()):
            return done
    return math.inf


def rskelf(A, x, occ, rank_or_tol, pxyfun=None, opts=None):
    """F = rskelf(A, x, occ, rank_or_tol, pxyfun, opts)   rskelf/rskelf.m:109-309.

    ``opts["stop"]`` is a level count or, as in the reference, a predicate
    ``stop(levels_done, l)``."""
    _check_handles(A, pxyfun)
    if opts and callable(opts.get("stop")):
        opts = dict(opts, stop=_stop_levels(opts["stop"], x, occ, opts))
    ptr, d, N, keep_x = _points(x)
    o, keep = _c_opts(opts)
    ka = A.c_struct()
    px = (pxyfun or Proxy("none", 1)).c_struct()
    h = C.c_void_p()
    _lib.check(_lib.lib().flam_rskelf(C.c_void_p(ptr), d, N, C.byref(ka), float(occ), float(rank_or_tol),
                                      C.byref(px), C.byref(o), C.byref(h)))
    return Factor(h.value, 1)


def rskelf_batched(As, xs, occ, rank_or_tol, pxyfun=None, opts=None, sizes=None):
    """Many independent rskelf problems in one device pipeline (one launch per level step).

    ``xs`` is a list of d x N_i point arrays, or (with ``sizes``) one d x sum(N_i)
    column-major CUDA tensor of all instances' points, used in place."""
    if opts and callable(opts.get("stop")):
        raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: a stop predicate needs one problem (each instance has its "
                                "own tree); pass a level count")
    for A in As:
        _check_handles(A, pxyfun)
    if sizes is not None:
        N = np.asarray(sizes, dtype=np.int64)
        d = xs.shape[0]
        if _is_cuda_tensor(xs):
            if xs.stride(0) != 1:
                raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: x must be a column-major d x N tensor")
            X, xptr = xs, xs.data_ptr()
        else:
            X = np.asfortranarray(xs, dtype=np.float64)
            xptr = X.ctypes.data
        if int(N.sum()) != xs.shape[1]:
            raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: sizes do not add up to the points given")
    else:
        xs = [np.asfortranarray(x, dtype=np.float64) for x in xs]
        d = xs[0].shape[0]
        X = np.asfortranarray(np.concatenate(xs, axis=1))
        xptr = X.ctypes.data
        N = np.array([x.shape[1] for x in xs], dtype=np.int64)
    karr = (_lib.FlamKernel * len(As))(*[A.c_struct() for A in As])
    o, keep = _c_opts(opts)
    px = (pxyfun or Proxy("none", 1)).c_struct()
    h = C.c_void_p()
    _lib.check(_lib.lib().flam_rskelf_batched(len(As), xptr, d, N.ctypes.data_as(C.POINTER(C.c_int64)), karr,
                                              float(occ), float(rank_or_tol), C.byref(px), C.byref(o), C.byref(h)))
    F = Factor(h.value, len(As))
    F._sizes = [int(n) for n in N]
    return F


def _fresh_copy(X):
    """A new column-major copy of X (MATLAB value semantics: the input is never modified)."""
    if _is_cuda_tensor(X):
        import torch
        if X.dim() == 1:
            return X.clone()
        Y = torch.empty_strided(tuple(X.shape), (1, X.shape[0]), dtype=torch.float64, device=X.device)
        Y.copy_(X)
        return Y
    return np.array(X, dtype=np.float64, order="F", copy=True)


def rskelf_sv(F, X, trans="n"):
    """Y = rskelf_sv(F, X, trans): returns a new array (MATLAB value semantics)."""
    return F.sv_(_fresh_copy(X), trans)


def rskelf_mv(F, X, trans="n"):
    """Y = rskelf_mv(F, X, trans): returns a new array."""
    return F.mv_(_fresh_copy(X), trans)


def matvec(F, X):
    """Y = A X with the FP64 registry matrix of F (an O(N^2) product evaluated on the fly)."""
    return F.matvec_(X, _fresh_copy(X))


def rskelf_ir_sv(F, B, ir_tol=1e-10, max_iter=10):
    """X = A \\ B by iterative refinement with F as the approximate inverse and the FP64
    residual B - A X.  Returns (X, refinement steps, per-column relative residuals)."""
    return F.ir_sv_(B, _fresh_copy(B), ir_tol, max_iter)


def rskelf_cholmv(F, X, trans="n"):
    """Y = C X (C' X for 't'/'c') with F = C C' (symm 'p').   rskelf/rskelf_cholmv.m:15-50."""
    return F._apply(_fresh_copy(X), trans, False, "flam_rskelf_cholmv")


def rskelf_cholsv(F, X, trans="n"):
    """Y = C \\ X (C' \\ X for 't'/'c') with F = C C' (symm 'p').   rskelf/rskelf_cholsv.m:15-50."""
    return F._apply(_fresh_copy(X), trans, True, "flam_rskelf_cholsv")


def rskelf_logdet(F):
    """log det of the factored matrix, imaginary part in [0, 2 pi).   rskelf/rskelf_logdet.m:11-33.

    A batched handle returns one value per instance."""
    n = F.ninst
    re = np.zeros(n)
    im = np.zeros(n)
    _lib.check(_lib.lib().flam_rskelf_logdet(F.handle, re.ctypes.data_as(C.POINTER(C.c_double)),
                                             im.ctypes.data_as(C.POINTER(C.c_double))))
    out = [complex(a, b) for a, b in zip(re, im)]
    return out[0] if n == 1 else out


def rskelf_diag(F, dinv=0):
    """D = rskelf_diag(F, dinv): diag(F) (dinv 0) or diag(inv(F)) (dinv 1), N values
    (all instances of a batched handle, in their concatenated order).
    rskelf/rskelf_diag.m:35-185, computed by unfolding box by box on the device."""
    D = np.zeros(F.info()["N"])
    _lib.check(_lib.lib().flam_rskelf_diag(F.handle, int(bool(dinv)), C.c_void_p(D.ctypes.data)))
    return D


def rskelf_spdiag(F, dinv=0):
    """D = rskelf_spdiag(F, dinv): the same diagonal as rskelf_diag (rskelf/rskelf_spdiag.m:19-85
    reaches it by sparse applies on unit vectors; the device unfolding gives the same values)."""
    return rskelf_diag(F, dinv)


def rskelf_partial_info(F, inst=0):
    """[Si, S] = rskelf_partial_info(F)   rskelf/rskelf_partial_info.m:12-20 (S: scipy CSC)."""
    return F.partial_info(inst)


def rskelf_partial_sv(F, X, svfun, trans="n"):
    """Upward sweep, X(Si,:) = svfun(X(Si,:), trans), downward sweep.   rskelf/rskelf_partial_sv.m:23-62.

    svfun gets a NumPy array for a NumPy X and a CUDA tensor for a CUDA X; trans is 'n' or 'c'.
    With several instances X(Si,:) stacks every instance's Si in instance order."""
    return F._partial(_fresh_copy(X), svfun, trans, True)


def rskelf_partial_mv(F, X, mvfun, trans="n"):
    """Upward sweep, X(Si,:) = mvfun(X(Si,:), trans), downward sweep.   rskelf/rskelf_partial_mv.m:23-62."""
    return F._partial(_fresh_copy(X), mvfun, trans, False)


class _DevBlock:
    """A column-major n x nrhs float64 block of device memory, seen through __cuda_array_interface__."""

    def __init__(self, ptr, n, nrhs):
        self.__cuda_array_interface__ = {"shape": (n, nrhs), "typestr": "<f8", "data": (ptr, False),
                                         "version": 2, "strides": (8, 8 * n)}


def factor_import(F, stream=None):
    """Device handle from a factorization in the reference's F layout (rskelf.m:157-159,
    249-257): a dict with N, symm and factors, each factor a dict of sk, rd (0-based), T,
    L, U, p, E, F (U, p, F unused for symm 'p').  Factorizations made elsewhere in rskelf
    format -- hifie2/hifie3, whose hifie_sv/mv are rskelf_sv/mv on that F
    (hifie/hifie_sv.m:21), or one saved from MATLAB -- then run rskelf_sv/mv/cholsv/cholmv/
    logdet on the device.  Factors act in list order."""
    symm = str(F["symm"]).lower()
    fs = F["factors"]
    chol = symm == "p"
    ks = np.array([len(f["sk"]) for f in fs], dtype=np.int64)
    rs = np.array([len(f["rd"]) for f in fs], dtype=np.int64)

    def cat(key, shape, dtype=np.float64):
        parts = []
        for f, k, r in zip(fs, ks, rs):
            a = np.asarray(f[key], dtype=dtype)
            parts.append(np.asfortranarray(a.reshape(shape(k, r))).ravel(order="F"))
        return np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(0, dtype))

    i64 = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))  # noqa: E731
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    sk = cat("sk", lambda k, r: (k,), np.int64)
    rd = cat("rd", lambda k, r: (r,), np.int64)
    T = cat("T", lambda k, r: (k, r))
    L = cat("L", lambda k, r: (r, r))
    E = cat("E", lambda k, r: (k, r))
    U = p = G = None
    if not chol:
        U = cat("U", lambda k, r: (r, r))
        p = cat("p", lambda k, r: (r,), np.int64)
        G = cat("F", lambda k, r: (r, k))
    h = C.c_void_p()
    nf = len(fs)
    z = np.zeros(1)
    zi = np.zeros(1, np.int64)
    _lib.check(_lib.lib().flam_factor_import(
        int(F["N"]), symm.encode()[:1], nf, i64(ks if nf else zi), i64(rs if nf else zi), i64(sk if sk.size else zi),
        i64(rd if rd.size else zi), dp(T if T.size else z), dp(L if L.size else z),
        None if U is None else dp(U if U.size else z), None if p is None else i64(p if p.size else zi),
        dp(E if E.size else z), None if G is None else dp(G if G.size else z), stream, C.byref(h)))
    out = Factor(h.value, 1)
    out._sizes = [int(F["N"])]
    return out


def hypoct(x, occ, lvlmax=math.inf, ext=None):
    """T = hypoct(x, occ, lvlmax, ext), built on the device.   core/hypoct.m:51-171."""
    x = np.asfortranarray(x, dtype=np.float64)
    d, N = x.shape
    e = None if ext is None or np.size(ext) == 0 else np.asfortranarray(ext, dtype=np.float64)
    lv = 0 if (lvlmax is None or lvlmax == math.inf) else int(lvlmax)
    if lv < 0 or (lvlmax is not None and lvlmax != math.inf and lvlmax < 1):
        raise _lib.FlamError(1, "FLAM:hypoct:invalidLvlmax: Maximum tree depth must be at least 1.")
    h = C.c_void_p()
    _lib.check(_lib.lib().flam_hypoct(x.ctypes.data, d, N, float(occ), lv, None if e is None else e.ctypes.data,
                                      None, C.byref(h)))
    F = Factor(h.value, 1)
    F._sizes = [N]
    return F


def id(A, rank_or_tol, Tmax=2.0, rrqr_iter=math.inf):  # noqa: A001 - the reference's name
    """[sk, rd, T, niter] = id(A, rank_or_tol, Tmax, rrqr_iter) on the device.   core/id.m:44-248."""
    A = np.asfortranarray(A, dtype=np.float64)
    m, n = A.shape
    k = C.c_int64()
    it = C.c_int64()
    perm = np.zeros(max(n, 1), np.int64)
    T = np.zeros(max(n * n // 4 + 1, 1))
    _lib.check(_lib.lib().flam_id(A.ctypes.data if A.size else None, m, n, max(m, 1), float(rank_or_tol), float(Tmax),
                                  -1 if rrqr_iter in (None, math.inf) else int(rrqr_iter), C.byref(k),
                                  perm.ctypes.data_as(C.POINTER(C.c_int64)), T.ctypes.data_as(C.POINTER(C.c_double)),
                                  C.byref(it)))
    kk = k.value
    Tm = T[:kk * (n - kk)].reshape(n - kk, kk).T.copy() if 0 < kk < n else np.zeros((kk, n - kk))
    return perm[:kk].copy(), perm[kk:n].copy(), Tm, it.value


def hypoct_perm(T):
    """P = hypoct_perm(T) for a handle returned by :func:`hypoct` or :func:`rskelf`."""
    return T.perm(0)


class Predictor:
    """Learned rank predictor (flam_predictor): a BF16 MLP 16 -> 128 -> 128 -> 1 trained and
    evaluated on the GPU by the library's own kernels.  Pass it as ``opts["predictor"]``
    together with ``opts["sketch"] = 1`` to size each box's sketch from its prediction."""

    NPARAM = 18817
    NFEAT = 16

    def __init__(self, seed=0, weights=None):
        h = C.c_void_p()
        _lib.check(_lib.lib().flam_predictor_create(int(seed), C.byref(h)))
        self.handle = h.value
        self._free = _lib.lib().flam_predictor_free
        if weights is not None:
            self.set_weights(weights)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self._free(h)
            self.handle = None

    @staticmethod
    def _f32(a, shape=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        if shape is not None and a.shape != shape:
            raise _lib.FlamError(1, f"FLAM:predictor:invalidArg: expected shape {shape}, got {a.shape}")
        return a

    def weights(self):
        w = np.zeros(self.NPARAM, np.float32)
        _lib.check(_lib.lib().flam_predictor_get(self.handle, w.ctypes.data_as(C.POINTER(C.c_float))))
        return w

    def set_weights(self, w):
        w = self._f32(w, (self.NPARAM,))
        _lib.check(_lib.lib().flam_predictor_set(self.handle, w.ctypes.data_as(C.POINTER(C.c_float))))

    def train(self, X, y, epochs=50, batch=256, lr=2e-3, seed=0):
        X = self._f32(X)
        y = self._f32(y)
        if X.ndim != 2 or X.shape[1] != self.NFEAT or y.shape != (X.shape[0],):
            raise _lib.FlamError(1, "FLAM:predictor:invalidArg: X must be n x 16 and y of length n")
        loss = C.c_float()
        fp = C.POINTER(C.c_float)
        _lib.check(_lib.lib().flam_predictor_train(self.handle, X.ctypes.data_as(fp), y.ctypes.data_as(fp),
                                                   X.shape[0], int(epochs), int(batch), float(lr), int(seed),
                                                   C.byref(loss)))
        return loss.value

    def predict(self, X):
        X = self._f32(X)
        out = np.zeros(max(X.shape[0], 1), np.float32)
        fp = C.POINTER(C.c_float)
        _lib.check(_lib.lib().flam_predictor_eval(self.handle, X.ctypes.data_as(fp), X.shape[0],
                                                  out.ctypes.data_as(fp)))
        return out[:X.shape[0]]

    def grad(self, X, y):
        """(mean squared error, its gradient) of one forward/backward pass on the GPU."""
        X = self._f32(X)
        y = self._f32(y)
        g = np.zeros(self.NPARAM, np.float32)
        loss = C.c_float()
        fp = C.POINTER(C.c_float)
        _lib.check(_lib.lib().flam_predictor_grad(self.handle, X.ctypes.data_as(fp), y.ctypes.data_as(fp),
                                                  X.shape[0], C.byref(loss), g.ctypes.data_as(fp)))
        return loss.value, g

    def save(self, path):
        np.savez_compressed(path, w=self.weights())

    @classmethod
    def load(cls, path):
        return cls(weights=np.load(path)["w"])


def _tune_dict(t):
    return {f: getattr(t, f) for f, _ in t._fields_}


def autotune(A, x, occ, rank_or_tol, pxyfun=None, opts=None, reps=2):
    """Measure the factorization's launch shapes on this problem (coordinate search over the
    row-split and shared-memory settings, device time) and keep the fastest for its class
    (dimension, kernel, log2 N) on the current device.  Returns the chosen setting."""
    _check_handles(A, pxyfun)
    xa = x if _is_cuda_tensor(x) else np.asfortranarray(x, dtype=np.float64)
    d, N = xa.shape
    o, keep = _c_opts(opts)
    px = (pxyfun or Proxy("none", 1)).c_struct()
    best = _lib.FlamTune()
    ptr = xa.data_ptr() if _is_cuda_tensor(xa) else xa.ctypes.data
    _lib.check(_lib.lib().flam_autotune(ptr, d, N, C.byref(A.c_struct()), float(occ), float(rank_or_tol), C.byref(px),
                                        C.byref(o), int(reps), C.byref(best)))
    return _tune_dict(best)


def tune_get(d, kernel, N):
    """The launch shapes factorizations of this class use on the current device."""
    t = _lib.FlamTune()
    _lib.check(_lib.lib().flam_tune_get(int(d), _kernel_id(kernel), int(N), C.byref(t)))
    return _tune_dict(t)


def tune_set(d, kernel, N, tune):
    """Install a saved tuning for this class on the current device."""
    t = _lib.FlamTune(**{k: int(v) for k, v in tune.items()})
    _lib.check(_lib.lib().flam_tune_set(int(d), _kernel_id(kernel), int(N), C.byref(t)))


def _kernel_id(kernel):
    from .registry import KERNELS
    return KERNELS[kernel] if isinstance(kernel, str) else int(kernel)
