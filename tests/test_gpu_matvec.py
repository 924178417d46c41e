"""FP64 on-the-fly products with the registry matrix (flam_matvec) and iterative
refinement on a loose factorization (flam_rskelf_ir_sv), against the dense FP64
matrix the oracle builds from the same registry entries (the reference's tests
form A*x from A(I,J): rskelf/test/ie_circle.m:47-48, ie_ellipse.m:51-80)."""
import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs

pytestmark = pytest.mark.gpu


def _cases():
    return {
        "star_w": (problems.star(2500, seed=1), configs.star(2500, seed=1), "n"),
        "ie_circle_dl": (problems.ie_circle(1500), configs.ie_circle(1500), "n"),
        "sphere": (problems.sphere(2200, p=64, seed=2), configs.sphere(2200, p=64, seed=2), "n"),
        "matern": (problems.matern_cube(1800, seed=3, p=32, p_rad=4), configs.matern_cube(1800, seed=3, p=32, p_rad=4),
                   "p"),
    }


@pytest.mark.parametrize("case", ["star_w", "ie_circle_dl", "sphere", "matern"])
@pytest.mark.parametrize("nrhs", [1, 5, 40, 100, 256])
def test_matvec_matches_dense_fp64(case, nrhs):
    (x, A, pxy), (xo, Ao, po), symm = _cases()[case]
    F = fb.rskelf(A, x, 64, 1e-6, pxy, dict(symm=symm))
    N = x.shape[1]
    rng = np.random.default_rng(nrhs)
    X = np.asfortranarray(rng.standard_normal((N, nrhs)))
    B = np.asfortranarray(rng.standard_normal((N, nrhs)))
    D = Ao.dense()
    Y = fb.matvec(F, X)
    ref = D @ X
    assert np.linalg.norm(Y - ref) <= 1e-13 * np.linalg.norm(ref) * np.sqrt(N)
    R = F.matvec_(X, np.asfortranarray(np.zeros((N, nrhs))), B=B)
    np.testing.assert_allclose(R, B - ref, rtol=0, atol=1e-12 * np.abs(ref).max() * np.sqrt(N))


def test_matvec_device_tensors_and_batched_handle():
    import torch
    sizes = [700, 1300, 950]
    xs, As, Aos = [], [], []
    for i, n in enumerate(sizes):
        x, A, pxy = problems.instance(n, 0.1 + 0.1 * i, 3 + i)
        xs.append(x)
        As.append(A)
        Aos.append(configs.star(n, a=0.1 + 0.1 * i, k=3 + i, clustered=False)[1])
    F = fb.rskelf_batched(As, xs, 64, 1e-6, pxy, dict(symm="n"))
    N = sum(sizes)
    X = torch.randn(N, 7, dtype=torch.float64, device="cuda").t().contiguous().t()
    Y = torch.empty_like(X)
    F.matvec_(X, Y)
    Xh, Yh = X.cpu().numpy(), Y.cpu().numpy()
    off = 0
    for n, Ao in zip(sizes, Aos):
        ref = Ao.dense() @ Xh[off:off + n]
        assert np.linalg.norm(Yh[off:off + n] - ref) <= 1e-13 * np.linalg.norm(ref) * np.sqrt(n)
        off += n


@pytest.mark.parametrize("case", ["star_w", "sphere"])
def test_refinement_reaches_fp64_tolerance_from_a_loose_factorization(case):
    (x, A, pxy), (xo, Ao, po), symm = _cases()[case]
    N = x.shape[1]
    B = np.asfortranarray(np.random.default_rng(4).standard_normal((N, 3)))
    D = Ao.dense()
    F = fb.rskelf(A, x, 64, 1e-4, pxy, dict(symm=symm))
    X0 = fb.rskelf_sv(F, B)
    r0 = np.linalg.norm(D @ X0 - B, axis=0) / np.linalg.norm(B, axis=0)
    X, it, rel = fb.rskelf_ir_sv(F, B, ir_tol=1e-11, max_iter=12)
    r = np.linalg.norm(D @ X - B, axis=0) / np.linalg.norm(B, axis=0)
    assert r0.max() > 1e-9 and it >= 1
    assert r.max() <= 1e-11
    np.testing.assert_allclose(rel, r, rtol=1e-2, atol=1e-15)
    np.testing.assert_allclose(X, np.linalg.solve(D, B), rtol=0, atol=1e-9 * np.abs(X).max())


def test_refinement_rejects_imported_factors_and_reports_non_convergence():
    x, A, pxy = problems.star(1500, seed=2)
    F = fb.rskelf(A, x, 64, 1e-3, pxy, dict(symm="n"))
    B = np.asfortranarray(np.random.default_rng(0).standard_normal((1500, 2)))
    with pytest.warns(UserWarning, match="notConverged"):
        X, it, rel = fb.rskelf_ir_sv(F, B, ir_tol=1e-14, max_iter=1)
    assert it == 1 and rel.max() > 1e-14
    fac = F.factors()
    G = fb.factor_import(fac)
    with pytest.raises(fb.FlamError, match="noMatrix"):
        fb.matvec(G, B)


def test_refinement_of_an_ill_conditioned_spd_matrix_converges():
    """Matern-3/2 covariance with a 1e-2 nugget (cond ~ 1e4): from a loose factorization the
    conjugate-gradient refinement of symm 'p' reaches 1e-10 where the stationary step would
    not contract."""
    x, A, pxy = problems.matern_cube(4000, seed=5, p=32, p_rad=4)
    xo, Ao, po = configs.matern_cube(4000, seed=5, p=32, p_rad=4)
    D = Ao.dense()
    F = fb.rskelf(A, x, 64, 1e-5, pxy, dict(symm="p", sketch=1))
    B = np.asfortranarray(np.random.default_rng(6).standard_normal((4000, 3)))
    X, it, rel = fb.rskelf_ir_sv(F, B, ir_tol=1e-10, max_iter=30)
    r = np.linalg.norm(D @ X - B, axis=0) / np.linalg.norm(B, axis=0)
    assert r.max() <= 1e-10 and it <= 30
    np.testing.assert_allclose(rel, r, rtol=1e-2, atol=1e-16)
