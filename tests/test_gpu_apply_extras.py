"""Cholesky half-applies, log-determinant and partial factorization on the device (GPU).

Two kinds of check:
* the device apply against the oracle's apply run on the SAME factors (exported
  from the device): this isolates the sweep kernels from the factorization, so
  the bar is rounding only (1e-12 relative);
* properties of the operator against the dense FP64 matrix: C C' = A,
  C \\ (C X) = X, logdet = slogdet(A), partial sv/mv with a dense skeleton
  solve = the full solve / multiply.
"""
import math

import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs
from oracle.rskelf import (rskelf as o_rskelf, rskelf_cholmv as o_cholmv, rskelf_cholsv as o_cholsv,
                           rskelf_logdet as o_logdet, rskelf_partial_info as o_pinfo, rskelf_sv as o_sv,
                           rskelf_mv as o_mv)

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def oracle_view(F, inst=0):
    """The device factors in the oracle's F layout (same sk/rd/T/L/U/p/E/F)."""
    d = F.factors(inst)
    return dict(N=d["N"], lvp=d["lvp"], factors=d["factors"], symm=d["symm"])


def dense_of(x, A):
    """Dense FP64 matrix of a registry kernel on points x (through the oracle's kernel)."""
    from oracle.registry import Kernel as OK
    return OK(A.kind, x, scale=A.scale, dval=A.dval, param=A.param, weights=A.weights).dense()


def spd_problem(N=2000):
    x, A, pxy = problems.circle(N)
    return x, A, pxy, configs.circle(N)[1].dense()


# ----------------------------------------------------------------- cholmv / cholsv
def test_cholmv_cholsv_match_oracle_on_device_factors():
    x, A, pxy, Ad = spd_problem(3000)
    F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="p"))
    Fo = oracle_view(F)
    B = np.asfortranarray(np.random.default_rng(2).standard_normal((3000, 5)))
    for trans in ("n", "t", "c"):
        assert rel(fb.rskelf_cholmv(F, B, trans), o_cholmv(Fo, B, trans)) < 1e-12
        assert rel(fb.rskelf_cholsv(F, B, trans), o_cholsv(Fo, B, trans)) < 1e-12
    # the full apply on the same factors too
    assert rel(fb.rskelf_sv(F, B), o_sv(Fo, B)) < 1e-12
    assert rel(fb.rskelf_mv(F, B), o_mv(Fo, B)) < 1e-12


def test_cholesky_factor_properties():
    N, tol = 1500, 1e-10
    x, A, pxy, Ad = spd_problem(N)
    F = fb.rskelf(A, x, 64, tol, pxy, dict(symm="p"))
    I = np.asfortranarray(np.eye(N))
    C = fb.rskelf_cholmv(F, I)                     # C
    Ct = fb.rskelf_cholmv(F, I, "c")               # C'
    np.testing.assert_allclose(Ct, C.T, rtol=0, atol=1e-12 * np.abs(C).max())
    assert rel(C @ C.T, Ad) < 1e2 * tol            # F = C C' approximates A
    B = np.asfortranarray(np.random.default_rng(3).standard_normal((N, 3)))
    assert rel(fb.rskelf_cholsv(F, fb.rskelf_cholmv(F, B)), B) < 1e-12
    assert rel(fb.rskelf_cholsv(F, fb.rskelf_cholmv(F, B, "c"), "c"), B) < 1e-12
    # mv = C (C' x), sv = C' \ (C \ x)
    assert rel(fb.rskelf_cholmv(F, fb.rskelf_cholmv(F, B, "c")), fb.rskelf_mv(F, B)) < 1e-12
    assert rel(fb.rskelf_cholsv(F, fb.rskelf_cholsv(F, B), "c"), fb.rskelf_sv(F, B)) < 1e-12


def test_chol_applies_need_symm_p():
    x, A, pxy = problems.star(1000, seed=1, clustered=False)
    F = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n"))
    B = np.asfortranarray(np.ones((1000, 1)))
    for fn, ident in ((fb.rskelf_cholmv, "FLAM:rskelf_cholmv:invalidSymm"),
                      (fb.rskelf_cholsv, "FLAM:rskelf_cholsv:invalidSymm")):
        with pytest.raises(fb.FlamError) as e:
            fn(F, B)
        assert e.value.identifier == ident
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf_sv(F, B, "x")
    assert e.value.identifier == "FLAM:chktrans:invalidTrans"


# ----------------------------------------------------------------- logdet
@pytest.mark.parametrize("case", ["n", "n_negative", "s", "p"])
def test_logdet(case):
    N, tol, symm = 2000, 1e-10, case[0]
    if case == "n":
        x, A, pxy = problems.star(N, seed=4, clustered=False)
        Ad = configs.star(N, seed=4, clustered=False)[1].dense()
    elif case == "n_negative":       # -I + K with N odd: det < 0, imaginary part pi
        N = 2001
        x, A0, pxy = problems.star(N, seed=4, clustered=False)
        A = fb.Kernel("laplace2d", scale=A0.scale, dval=-1.0, weights=A0.weights)
        Ad = dense_of(x, A)
    else:
        x, A, pxy, Ad = spd_problem(N)
    F = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm))
    ld = fb.rskelf_logdet(F)
    lo = o_logdet(oracle_view(F))
    assert abs(ld.real - lo.real) <= 1e-12 * max(1.0, abs(lo.real))
    # imaginary parts as angles: the oracle sums floating-point multiples of pi and can land
    # just below 2 pi where the exact answer (the device's: 0 or pi) is 0
    assert abs(np.exp(1j * ld.imag) - np.exp(1j * lo.imag)) < 1e-9
    assert 0 <= ld.imag < 2 * math.pi
    sign, la = np.linalg.slogdet(Ad)
    assert abs(ld.real - la) < 1e-8 * max(1.0, abs(la))
    assert abs(np.exp(1j * ld.imag) - sign) < 1e-9
    if case == "n_negative":
        assert sign < 0 and abs(ld.imag - math.pi) < 1e-12


def test_logdet_batched_per_instance():
    Ns, aa, kk = problems.instance_batch(4, seed=2, nmin=500, nmax=1500)
    items = [problems.instance(int(n), a, k) for n, a, k in zip(Ns, aa, kk)]
    Fb = fb.rskelf_batched([it[1] for it in items], [it[0] for it in items], 64, 1e-10, items[0][2])
    lds = fb.rskelf_logdet(Fb)
    assert len(lds) == 4
    for i, (x, A, pxy) in enumerate(items):
        F = fb.rskelf(A, x, 64, 1e-10, pxy)
        assert abs(fb.rskelf_logdet(F) - lds[i]) < 1e-12 * max(1.0, abs(lds[i]))


# ----------------------------------------------------------------- partial factorization
def test_partial_info_matches_oracle():
    N, tol = 4000, 1e-10
    x, A, pxy = problems.star(N, seed=5, clustered=False)
    xo, Ao, po = configs.star(N, seed=5, clustered=False)
    for stop in (1, 2, 3):
        F = fb.rskelf(A, x, 64, tol, pxy, dict(symm="n", stop=stop))
        Fo = o_rskelf(Ao, xo, 64, tol, po, dict(symm="n", stop=stop), order="level_sync")
        Si, S = fb.rskelf_partial_info(F)
        Sio, So = o_pinfo(Fo)
        np.testing.assert_array_equal(Si, Sio)
        assert F.info()["nrem"] == len(Si)
        Sd = S.toarray()
        # S is block diagonal over boxes: its pattern is the oracle's nonzero pattern
        np.testing.assert_array_equal(Sd != 0, So != 0)
        # the values follow T = R11 \ R12, whose rounding grows with cond(R11) (up to
        # 1/tol): two correct factorizations with the same skeletons agree to about
        # eps / tol, not to eps
        assert np.abs(Sd - So).max() <= 1e-6 * np.abs(So).max()
        if stop == 1:
            # one level: every leaf's block is -E G of its own factor, so S is fixed by the
            # device's exported factors up to rounding (rskelf.m:245-246, 296-306)
            pos = {int(g): q for q, g in enumerate(Si)}
            Se = np.zeros_like(Sd)
            for f in F.factors()["factors"]:
                ix = [pos[int(g)] for g in f["sk"]]
                Se[np.ix_(ix, ix)] = -(f["E"] @ f["F"])
            assert np.abs(Sd - Se).max() <= 1e-13 * np.abs(Se).max()


def test_partial_sv_mv_with_dense_skeleton_system():
    N, tol = 3000, 1e-10
    x, A, pxy = problems.star(N, seed=6, clustered=False)
    Ad = configs.star(N, seed=6, clustered=False)[1].dense()
    B = np.asfortranarray(np.random.default_rng(7).standard_normal((N, 3)))
    Xfull = np.linalg.solve(Ad, B)
    for stop in (0, 2, 4):
        F = fb.rskelf(A, x, 64, tol, pxy, dict(symm="n", stop=stop))
        Si, S = fb.rskelf_partial_info(F)
        Ssys = Ad[np.ix_(Si, Si)] + S.toarray()
        if stop == 0:
            assert len(Si) == N and S.nnz == 0
        calls = []

        def svfun(Y, trans):
            calls.append(trans)
            return np.linalg.solve(Ssys if trans == "n" else Ssys.T, Y)

        def mvfun(Y, trans):
            return (Ssys if trans == "n" else Ssys.T) @ Y

        for trans in ("n", "t"):
            Op = Ad if trans == "n" else Ad.T
            X = fb.rskelf_partial_sv(F, B, svfun, trans)
            assert rel(Op @ X, B) < 1e3 * tol, (stop, trans)
            Y = fb.rskelf_partial_mv(F, B, mvfun, trans)
            assert rel(Y, Op @ B) < 1e3 * tol, (stop, trans)
            if trans == "n":
                assert rel(X, Xfull) < 1e3 * tol
        assert calls == ["n", "c"]


def test_partial_on_device_tensors_and_callback_errors():
    import torch
    N, tol = 2500, 1e-10
    x, A, pxy, Ad = spd_problem(N)
    F = fb.rskelf(A, x, 64, tol, pxy, dict(symm="p", stop=2))
    Si, S = fb.rskelf_partial_info(F)
    Ssys = torch.from_numpy(Ad[np.ix_(Si, Si)] + S.toarray()).cuda()
    B = torch.randn(N, 2, dtype=torch.float64, device="cuda").t().contiguous().t()
    seen = []

    def svfun(Y, trans):
        seen.append(type(Y))
        return torch.linalg.solve(Ssys, Y)

    X = fb.rskelf_partial_sv(F, B, svfun)
    assert seen == [torch.Tensor]
    assert rel(Ad @ X.cpu().numpy(), B.cpu().numpy()) < 1e3 * tol

    def bad(Y, trans):
        raise ArithmeticError("skeleton solve failed")

    with pytest.raises(ArithmeticError):
        fb.rskelf_partial_sv(F, B, bad)
    X2 = fb.rskelf_partial_sv(F, B, svfun)          # the handle is still usable
    assert torch.equal(X, X2)


def test_partial_batched_stacks_instances():
    Ns, aa, kk = problems.instance_batch(3, seed=4, nmin=1500, nmax=2500)
    items = [problems.instance(int(n), a, k) for n, a, k in zip(Ns, aa, kk)]
    Fb = fb.rskelf_batched([it[1] for it in items], [it[0] for it in items], 64, 1e-10, items[0][2],
                           dict(stop=2))
    B = np.asfortranarray(np.random.default_rng(1).standard_normal((int(Ns.sum()), 2)))
    blocks, off = [], 0
    for i, (x, A, pxy) in enumerate(items):
        F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(stop=2))
        Si, S = fb.rskelf_partial_info(F)
        Sib, Sb = Fb.partial_info(i)
        np.testing.assert_array_equal(Si, Sib)
        # a batch shares the levels with other instances, so the row-split form of the
        # few-box levels can differ from the single run: S agrees to eps / tol
        Sd, Sbd = S.toarray(), Sb.toarray()
        np.testing.assert_array_equal(Sd != 0, Sbd != 0)
        assert np.abs(Sd - Sbd).max() <= 1e-6 * np.abs(Sd).max()
        Ad = dense_of(x, A)
        blocks.append(Ad[np.ix_(Si, Si)] + S.toarray())
        off += x.shape[1]
    sizes = [b.shape[0] for b in blocks]

    def svfun(Y, trans):
        out, o = np.empty_like(Y), 0
        for Bk, n in zip(blocks, sizes):
            out[o:o + n] = np.linalg.solve(Bk, Y[o:o + n])
            o += n
        return out

    X = fb.rskelf_partial_sv(Fb, B, svfun)
    off = 0
    for i, (x, A, pxy) in enumerate(items):
        n = x.shape[1]
        Ad = dense_of(x, A)
        assert rel(Ad @ X[off:off + n], B[off:off + n]) < 1e-7
        off += n
