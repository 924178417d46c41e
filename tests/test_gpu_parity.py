"""Device path against the oracle (GPU).

Parity bar:
* hypoct / hypoct_perm: bit-exact (every array, every box);
* id: same rank and same skeleton set, |T| <= Tmax, interpolation error within
  the tolerance;
* rskelf: same tree, same per-box rank and skeleton set as the oracle's
  level-synchronous order on non-symmetric geometries, same level table;
  sv / mv within 1e3 * tol of the oracle's and of the dense FP64 operator.
  (Pivot ORDER inside a skeleton set can differ where trailing column norms
  tie to rounding; the set and the factorization do not.)
"""
import math
import os

import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs
from oracle.idecomp import id_
from oracle.rskelf import rskelf as o_rskelf, rskelf_mv as o_mv, rskelf_sv as o_sv
from oracle.tree import hypoct as o_hypoct, hypoct_perm as o_perm, tree_arrays

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def tree_equal(T, t):
    assert T["nlvl"] == t["nlvl"]
    np.testing.assert_array_equal(T["lvp"], t["lvp"])
    np.testing.assert_array_equal(T["l"], t["l"])
    np.testing.assert_array_equal(T["ctr"], t["ctr"])
    np.testing.assert_array_equal(T["prnt"], t["prnt"])
    for key in ("chld", "nbor", "xi"):
        assert len(T[key]) == len(t[key])
        for a, b in zip(T[key], t[key]):
            np.testing.assert_array_equal(a, b)


# ----------------------------------------------------------------- tree (K1/K2)
@pytest.mark.parametrize("case", ["ie_circle", "star", "sphere", "cube", "lvlmax", "ext", "tiny"])
def test_tree_bit_exact(case):
    kw = {}
    if case == "ie_circle":
        x, occ = problems.ie_circle(16384)[0], 64
    elif case == "star":
        x, occ = problems.star(30000, seed=3)[0], 64
    elif case == "sphere":
        x, occ = problems.sphere(20000, seed=1)[0], 64
    elif case == "cube":
        x, occ = np.random.default_rng(5).random((3, 6000)), 24
    elif case == "lvlmax":
        x, occ, kw = problems.star(8000, seed=9)[0], 16, dict(lvlmax=4)
    elif case == "ext":
        x, occ, kw = problems.circle(3000)[0], 32, dict(ext=np.array([[-2.0, 2.0], [-1.5, 1.5]]))
    else:
        x, occ = np.array([[0.0, 1.0, 0.0, 1.0, 0.3], [0.0, 0.0, 1.0, 1.0, 0.6]]), 1
    H = fb.hypoct(x, occ, **kw)
    t = o_hypoct(x, occ, **kw)
    tree_equal(H.tree(), t)
    np.testing.assert_array_equal(H.perm(), o_perm(t))


@pytest.mark.parametrize("name", ["tree_star3000.npz", "tree_cube2000.npz", "tree_sphere4000_lvlmax3.npz"])
def test_tree_golden(name):
    g = np.load(os.path.join(GOLD, name))
    kw = {} if not np.isfinite(g["lvlmax"]) else dict(lvlmax=int(g["lvlmax"]))
    H = fb.hypoct(g["x"], int(g["occ"]), **kw)
    T = H.tree()
    np.testing.assert_array_equal(T["lvp"], g["lvp"])
    np.testing.assert_array_equal(T["ctr"], g["ctr"])
    np.testing.assert_array_equal(np.concatenate([a for a in T["nbor"] if len(a)]), g["nbor"])
    np.testing.assert_array_equal(np.concatenate([a for a in T["xi"] if len(a)]), g["xi"])
    np.testing.assert_array_equal(H.perm(), g["perm"])


# ----------------------------------------------------------------- id (K5/K6)
def test_id_golden_cases():
    g = np.load(os.path.join(GOLD, "id_cases.npz"))
    for c in range(6):
        A = g[f"A{c}"]
        rot, Tmax = g[f"p{c}"]
        sk, rd, T, it = fb.id(A, rot, Tmax)
        assert len(sk) == len(g[f"sk{c}"]), c
        if rot < 1 or g[f"it{c}"] == 0:
            # tolerance mode is invariant under the QR's row signs: same skeleton set.
            # The fixed-rank branch with swaps (id.m:168-198) depends on those signs
            # (R(k+1,k+1) = sqrt(c2(1))); there the ID properties are checked instead.
            assert set(sk.tolist()) == set(g[f"sk{c}"].tolist()), c
        if T.size:
            assert np.abs(T).max() <= Tmax * (1 + 1e-9), c
            err = np.linalg.norm(A[:, rd] - A[:, sk] @ T, 2) / np.linalg.norm(A, 2)
            tol = math.fmod(rot, 1.0) or 1e-12
            ref = np.linalg.norm(A[:, g[f"rd{c}"]] - A[:, g[f"sk{c}"]] @ g[f"T{c}"], 2) / np.linalg.norm(A, 2)
            assert err <= max(10 * ref, 100 * tol), (c, err, ref)


def test_id_edge_cases():
    sk, rd, T, _ = fb.id(np.zeros((0, 6)), 1e-6)
    assert len(sk) == 0 and list(rd) == list(range(6))
    sk, rd, T, _ = fb.id(np.ones((5, 1)), 1e-6)
    assert list(sk) == [0] and len(rd) == 0
    A = np.outer(np.arange(1.0, 9.0), [1.0, 2.0, 3.0])
    sk, rd, T, _ = fb.id(A, 1e-9)
    assert list(sk) == [2] and np.allclose(A[:, rd], A[:, sk] @ T)
    B = np.random.default_rng(0).standard_normal((30, 200))   # n > 128: global-memory work matrices
    sk, rd, T, _ = fb.id(B, 1e-10)
    sk0, rd0, T0, _ = id_(B, 1e-10)
    assert set(sk.tolist()) == set(sk0.tolist())


# ----------------------------------------------------------------- rskelf
def compare_factor(F, Fo, need_sets=1.0):
    fg = F.factors()
    fs, fo = fg["factors"], Fo["factors"]
    assert len(fs) == len(fo)
    np.testing.assert_array_equal(fg["lvp"], Fo["lvp"])
    assert [len(a["sk"]) for a in fs] == [len(b["sk"]) for b in fo]
    same = sum(set(a["sk"].tolist()) == set(b["sk"].tolist()) for a, b in zip(fs, fo))
    assert same >= need_sets * len(fs), (same, len(fs))
    rows = F.level_stats()
    np.testing.assert_array_equal(rows, [[s["lvl"], s["nblk"], s["nrem1"], s["nrem2"]] for s in Fo["stats"]])


@pytest.mark.parametrize("symm", ["n", "s", "p"])
def test_rskelf_matches_oracle(symm):
    N, tol = 3000, 1e-10
    if symm == "n":
        x, A, pxy = problems.star(N, seed=5, clustered=False)
        xo, Ao, po = configs.star(N, seed=5, clustered=False)
    else:
        x, A, pxy = problems.circle(N)
        xo, Ao, po = configs.circle(N)
    F = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm))
    Fo = o_rskelf(Ao, xo, 64, tol, po, dict(symm=symm), order="level_sync")
    # the circle is symmetric: exact column-norm ties make skeleton choice order-dependent
    compare_factor(F, Fo, need_sets=1.0 if symm == "n" else 0.0)
    Ad = Ao.dense()
    B = np.asfortranarray(np.random.default_rng(3).standard_normal((N, 4)))
    for trans in ("n", "t", "c"):
        Op = Ad if trans == "n" else Ad.T
        X = fb.rskelf_sv(F, B, trans)
        assert np.linalg.norm(Op @ X - B) / np.linalg.norm(B) < 1e3 * tol
        Y = fb.rskelf_mv(F, B, trans)
        assert np.linalg.norm(Op @ B - Y) / np.linalg.norm(Op @ B) < 1e3 * tol
        Xo = o_sv(Fo, B, trans)
        assert np.linalg.norm(X - Xo) / np.linalg.norm(Xo) < 1e3 * tol
        Yo = o_mv(Fo, B, trans)
        assert np.linalg.norm(Y - Yo) / np.linalg.norm(Yo) < 1e3 * tol


def test_rskelf_golden_star():
    g = np.load(os.path.join(GOLD, "rskelf_star2048_n.npz"))
    x, A, pxy = problems.star(2048, seed=7, clustered=False)
    np.testing.assert_array_equal(x, g["x"])
    F = fb.rskelf(A, x, 64, float(g["tol"]), pxy, dict(symm="n"))
    fs = F.factors()["factors"]
    np.testing.assert_array_equal([len(f["sk"]) for f in fs], g["k"])
    np.testing.assert_array_equal(np.concatenate([np.sort(f["sk"]) for f in fs]), g["sk_sorted"])
    np.testing.assert_array_equal(F.level_stats(), g["stats"])
    X = fb.rskelf_sv(F, np.asfortranarray(g["B"]))
    assert np.linalg.norm(X - g["X"]) / np.linalg.norm(g["X"]) < 1e-8
    Y = fb.rskelf_mv(F, np.asfortranarray(g["B"]))
    assert np.linalg.norm(Y - g["Y"]) / np.linalg.norm(g["Y"]) < 1e-8


def test_rskelf_golden_circle_chol():
    g = np.load(os.path.join(GOLD, "rskelf_circle2048_p.npz"))
    x, A, pxy = problems.circle(2048)
    F = fb.rskelf(A, x, 64, float(g["tol"]), pxy, dict(symm="p"))
    np.testing.assert_array_equal(F.level_stats()[:, :3], g["stats"][:, :3])
    X = fb.rskelf_sv(F, np.asfortranarray(g["B"]))
    assert np.linalg.norm(X - g["X"]) / np.linalg.norm(g["X"]) < 1e-8


def test_rskelf_clustered_and_rrqr():
    # uneven boxes (Beta-clustered curve) and Tmax close to 1, so RRQR swaps happen
    N, tol = 4000, 1e-10
    x, A, pxy = problems.star(N, seed=8)
    xo, Ao, po = configs.star(N, seed=8)
    for Tmax in (2.0, 1.05):
        F = fb.rskelf(A, x, 32, tol, pxy, dict(symm="n", Tmax=Tmax))
        Fo = o_rskelf(Ao, xo, 32, tol, po, dict(symm="n", Tmax=Tmax), order="level_sync")
        compare_factor(F, Fo, need_sets=0.97)
        for f in F.factors()["factors"]:
            if f["T"].size:
                assert np.abs(f["T"]).max() <= Tmax * (1 + 1e-9)
        Ad = Ao.dense()
        B = np.asfortranarray(np.random.default_rng(1).standard_normal((N, 2)))
        assert np.linalg.norm(Ad @ fb.rskelf_sv(F, B) - B) / np.linalg.norm(B) < 1e3 * tol


def test_rskelf_fixed_rank_and_options():
    x, A, pxy = problems.star(2500, seed=6, clustered=False)
    xo, Ao, po = configs.star(2500, seed=6, clustered=False)
    Ad = Ao.dense()
    B = np.asfortranarray(np.random.default_rng(4).standard_normal((2500, 2)))
    for rot, opts in [(20.0, dict(Tmax=1.05)), (20.0, dict(Tmax=math.inf)), (1e-8, dict(Tmax=math.inf)),
                      (1e-8, dict(rrqr_iter=0)), (1e-8, dict(lvlmax=3))]:
        F = fb.rskelf(A, x, 64, rot, pxy, dict(symm="n", **opts))
        Fo = o_rskelf(Ao, xo, 64, rot, po, dict(symm="n", **opts), order="level_sync")
        X = fb.rskelf_sv(F, B)
        Xo = o_sv(Fo, B)
        if rot >= 1 and opts.get("Tmax") != math.inf:
            # fixed rank with RRQR swaps: the reference update (id.m:168-198) depends on the
            # QR's row signs, so compare ranks and the quality of the factorization only
            compare_factor(F, Fo, need_sets=0.0)
            ro = np.linalg.norm(Ad @ Xo - B) / np.linalg.norm(B)
            rg = np.linalg.norm(Ad @ X - B) / np.linalg.norm(B)
            assert rg < 10 * ro + 1e-12, (rg, ro)
        else:
            compare_factor(F, Fo, need_sets=0.97)
            assert np.linalg.norm(X - Xo) / np.linalg.norm(Xo) < 1e-6


def test_rskelf_partial_factorization():
    x, A, pxy = problems.circle(4096)
    F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(stop=2))
    info = F.info()
    Fo = o_rskelf(configs.circle(4096)[1], x, 64, 1e-10, configs.circle(4096)[2], dict(stop=2), order="level_sync")
    assert info["nstep"] == 2 and info["nrem"] == len(Fo["Si"])


def test_rskelf_small_problems():
    for N in (1, 2, 5, 63, 64, 65):
        x, A, pxy = problems.circle(N)
        F = fb.rskelf(A, x, 64, 1e-10, pxy)
        Ad = configs.circle(N)[1].dense()
        B = np.asfortranarray(np.random.default_rng(N).standard_normal((N, 3)))
        X = fb.rskelf_sv(F, B)
        assert np.linalg.norm(Ad @ X - B) / np.linalg.norm(B) < 1e-10, N


@pytest.mark.parametrize("case", ["sphere", "matern", "gaussian"])
def test_rskelf_3d_and_covariance(case):
    if case == "sphere":
        x, A, pxy = problems.sphere(6000, p=256, seed=2)
        xo, Ao, po = configs.sphere(6000, p=256, seed=2)
        symm, tol, occ = "n", 1e-8, 64
    elif case == "matern":
        x, A, pxy = problems.matern_cube(5000, seed=1, p=64, p_rad=6)
        xo, Ao, po = configs.matern_cube(5000, seed=1, p=64, p_rad=6)
        symm, tol, occ = "p", 1e-6, 64
    else:
        th = np.arange(1, 3001) * 2 * math.pi / 3000
        x = np.stack([np.cos(th), np.sin(th)])
        A = fb.Kernel("gaussian", dval=1.0 + 1e-4, param=100.0)
        pxy = fb.Proxy("annulus", 16, "gaussian", param=100.0, p_rad=16)
        from oracle.registry import Kernel as OK, Proxy as OP
        xo, Ao = x, OK("gaussian", x, dval=1.0 + 1e-4, param=100.0)
        po = OP("annulus", 2, 16, "gaussian", param=100.0, p_rad=16)
        symm, tol, occ = "p", 1e-10, 64
    # two factorizations within tol of A give solutions within cond(A) * tol of each
    # other; the Gaussian matrix's diagonal shift 1e-4 puts cond(A) near 1e4
    amp = 1e4 if case == "gaussian" else 1e3
    F = fb.rskelf(A, x, occ, tol, pxy, dict(symm=symm))
    Fo = o_rskelf(Ao, xo, occ, tol, po, dict(symm=symm), order="level_sync")
    assert [len(f["sk"]) for f in F.factors()["factors"]] == [len(f["sk"]) for f in Fo["factors"]] or \
        abs(F.info()["nfactor"] - len(Fo["factors"])) <= 1
    N = x.shape[1]
    B = np.asfortranarray(np.random.default_rng(6).standard_normal((N, 2)))
    X = fb.rskelf_sv(F, B)
    Xo = o_sv(Fo, B)
    assert np.linalg.norm(X - Xo) / np.linalg.norm(Xo) < amp * tol
    Ad = Ao.dense()
    assert np.linalg.norm(Ad @ X - B) / np.linalg.norm(B) < 1e4 * tol


def test_not_positive_definite_is_reported():
    x, A, pxy = problems.circle(2048)
    bad = fb.Kernel("laplace2d", scale=2 * math.pi / 2048, dval=-1.0)   # indefinite diagonal
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf(bad, x, 64, 1e-10, pxy, dict(symm="p"))
    assert e.value.identifier == "FLAM:rskelf:notPosDef"
    F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="p"))    # the context is still usable
    assert F.info()["nfactor"] > 0


def test_batched_equals_single():
    # The same boxes get the same ID and elimination in a batch as alone; only the
    # row-split form of the few-box levels (which depends on how many boxes share a
    # level) changes the rounding of R, hence T up to rounding and near-tied pivots.
    Ns, aa, kk = problems.instance_batch(6, seed=1, nmin=600, nmax=3000)
    items = [problems.instance(int(n), a, k) for n, a, k in zip(Ns, aa, kk)]
    Fb = fb.rskelf_batched([it[1] for it in items], [it[0] for it in items], 64, 1e-10, items[0][2])
    B = np.asfortranarray(np.random.default_rng(0).standard_normal((int(Ns.sum()), 2)))
    Xb = fb.rskelf_sv(Fb, B)
    off = 0
    for i, (x, A, pxy) in enumerate(items):
        F = fb.rskelf(A, x, 64, 1e-10, pxy)
        fs, fbs = F.factors()["factors"], Fb.factors(i)["factors"]
        assert len(fs) == len(fbs)
        same = sum(set(a["sk"].tolist()) == set(b["sk"].tolist()) for a, b in zip(fs, fbs))
        assert same >= 0.97 * len(fs), (same, len(fs))
        for a, b in zip(fs, fbs):
            if set(a["sk"].tolist()) == set(b["sk"].tolist()) and set(a["rd"].tolist()) == set(b["rd"].tolist()):
                ia, ib = np.argsort(a["rd"]), np.argsort(b["rd"])
                ja, jb = np.argsort(a["sk"]), np.argsort(b["sk"])
                if a["T"].size:
                    Ta, Tb = a["T"][np.ix_(ja, ia)], b["T"][np.ix_(jb, ib)]
                    assert np.abs(Ta - Tb).max() <= 1e-5 * max(1.0, np.abs(Tb).max())
        Xi = fb.rskelf_sv(F, np.asfortranarray(B[off:off + x.shape[1]]))
        Xs = Xb[off:off + x.shape[1]]
        assert np.linalg.norm(Xi - Xs) / np.linalg.norm(Xs) < 1e-8
        off += x.shape[1]


def test_device_tensors():
    import torch
    x, A, pxy = problems.star(5000, seed=2)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().t()
    Ad = fb.Kernel("laplace2d", weights=torch.from_numpy(A.weights).cuda())
    F1 = fb.rskelf(A, x, 64, 1e-10, pxy)
    F2 = fb.rskelf(Ad, xd, 64, 1e-10, pxy)
    B = torch.randn(5000, 3, dtype=torch.float64, device="cuda").t().contiguous().t()
    B0 = B.clone()
    X2 = fb.rskelf_sv(F2, B)
    assert torch.equal(B, B0)                        # value semantics: the input is untouched
    X1 = fb.rskelf_sv(F1, np.asfortranarray(B.cpu().numpy()))
    np.testing.assert_array_equal(X2.cpu().numpy(), X1)


def test_host_buffers_many_rhs_match_device():
    # 64 or more right-hand sides in host memory go through the overlapped copy path
    # (two column halves); every column is computed as on the device path
    import torch
    x, A, pxy = problems.star(5000, seed=4)
    F = fb.rskelf(A, x, 64, 1e-10, pxy)
    B = np.asfortranarray(np.random.default_rng(9).standard_normal((5000, 97)))
    for fn, inplace in ((fb.rskelf_sv, F.sv_), (fb.rskelf_mv, F.mv_)):
        Xh = fn(F, B)                                              # pageable host memory
        P = torch.empty((97, 5000), dtype=torch.float64).pin_memory()
        P.copy_(torch.from_numpy(B.T.copy()))
        Xp = inplace(P.t().numpy())                                # pinned, in place
        Xd = fn(F, torch.from_numpy(B.T.copy()).cuda().t()).cpu().numpy()
        np.testing.assert_array_equal(Xh, Xd)
        np.testing.assert_array_equal(Xp, Xd)
