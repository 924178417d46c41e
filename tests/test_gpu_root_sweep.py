"""Grid-wide solve sweeps of large root factors (GPU).

A factor with no skeletons (k = 0) and r >= 1024 redundant rows -- the root of a
problem that stops with a large block -- is swept across the whole GPU (blocked
triangular solves with FP64 tensor-path updates) instead of by one CTA per
right-hand-side tile.  The sweeps of rskelf_sv.m / rskelf_cholsv.m (op 'n', 't', 'c';
symm 'n', 's', 'p') are checked against the oracle's apply on the SAME factors
exported from the device (rounding only), and the solves against the dense matrix.
"""
import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs
from oracle.rskelf import rskelf_cholsv as o_cholsv, rskelf_mv as o_mv, rskelf_sv as o_sv

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def oracle_view(F):
    d = F.factors(0)
    return dict(N=d["N"], lvp=d["lvp"], factors=d["factors"], symm=d["symm"])


def root_r(F):
    return max((len(f["rd"]) for f in F.factors(0)["factors"] if len(f["sk"]) == 0), default=0)


def _problem(symm, N):
    if symm == "n":
        x, A, pxy = problems.star(N, seed=3)
        return x, A, pxy, configs.star(N, seed=3)[1].dense()
    x, A, pxy = problems.circle(N)
    return x, A, pxy, configs.circle(N)[1].dense()


@pytest.mark.parametrize("symm", ["n", "s", "p"])
@pytest.mark.parametrize("nrhs", [1, 37, 300])
def test_single_box_root_matches_oracle_and_dense(symm, nrhs):
    """occ >= N: the whole problem is one dense LU (or Cholesky) factor of r = N."""
    N = 1500
    x, A, pxy, D = _problem(symm, N)
    F = fb.rskelf(A, x, 4096, 1e-10, pxy, dict(symm=symm))
    assert root_r(F) == N
    Fo = oracle_view(F)
    B = np.asfortranarray(np.random.default_rng(nrhs).standard_normal((N, nrhs)))
    for trans in ("n", "t", "c"):
        Y = fb.rskelf_sv(F, B, trans)
        assert rel(Y, o_sv(Fo, B, trans)) < 1e-12
        Dt = D if trans == "n" else D.T
        assert rel(Dt @ Y, B) < 1e-10
        assert rel(fb.rskelf_mv(F, B, trans), o_mv(Fo, B, trans)) < 1e-12
        if symm == "p":
            assert rel(fb.rskelf_cholsv(F, B, trans), o_cholsv(Fo, B, trans)) < 1e-12


@pytest.mark.parametrize("symm", ["n", "p"])
def test_compressed_problem_with_large_root(symm):
    """A multi-level factorization that stops with a root block above 1024 rows."""
    N = 12000
    if symm == "n":
        x, A, pxy = problems.sphere(N, p=64, seed=4)
        D = configs.sphere(N, p=64, seed=4)[1].dense()
    else:
        x, A, pxy = problems.matern_cube(N, seed=4, p=32, p_rad=4)
        D = configs.matern_cube(N, seed=4, p=32, p_rad=4)[1].dense()
    F = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm=symm))
    assert root_r(F) >= 1024
    Fo = oracle_view(F)
    B = np.asfortranarray(np.random.default_rng(1).standard_normal((N, 64)))
    for trans in ("n", "t"):
        Y = fb.rskelf_sv(F, B, trans)
        assert rel(Y, o_sv(Fo, B, trans)) < 1e-11
    Y = fb.rskelf_sv(F, B)
    assert rel(D @ Y, B) < 1e-6


def test_large_root_under_graph_replay_and_refinement():
    """Repeated applies on the same device buffers are captured and replayed as a CUDA
    graph that holds the grid-wide root sweep; refinement uses the same sweeps."""
    import torch
    N = 1500
    x, A, pxy, D = _problem("n", N)
    F = fb.rskelf(A, x, 4096, 1e-10, pxy, dict(symm="n"))
    B = np.random.default_rng(9).standard_normal((N, 48))
    ref = np.linalg.solve(D, B)
    Bd = torch.from_numpy(B.T.copy()).cuda().t()
    Xd = torch.empty_like(Bd)
    r0 = F.profile()["graph_replays"]
    for _ in range(4):
        Xd.copy_(Bd)
        F.sv_(Xd)
        torch.cuda.synchronize()
        assert rel(Xd.cpu().numpy(), ref) < 1e-10
    assert F.profile()["graph_replays"] - r0 == 3
    X, it, rr = fb.rskelf_ir_sv(F, np.asfortranarray(B), ir_tol=1e-13, max_iter=3)
    assert rel(X, ref) < 1e-10
