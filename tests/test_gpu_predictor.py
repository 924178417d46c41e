"""The learned rank predictor: its GPU training kernels against the NumPy oracle
(gradient check), training on ranks logged by the exact ID, and what it gains in the
sketched compression -- fewer sketch rows at the same FP64 error after refinement,
with the exact ID (core/id.m) as the fallback when a prediction is too low."""
import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs, mlp

pytestmark = pytest.mark.gpu


def test_gradient_matches_numpy_oracle():
    P = fb.Predictor(seed=3)
    w = P.weights()
    rng = np.random.default_rng(1)
    X = rng.random((300, 16)).astype(np.float32)
    y = rng.random(300).astype(np.float32)
    loss, g = P.grad(X, y)
    lo, go = mlp.loss_and_grad(w, X, y)
    assert abs(loss - lo) <= 1e-4 * max(lo, 1e-6)
    offs = np.cumsum([0, 128 * 16, 128, 128 * 128, 128, 128, 1])
    for a, b in zip(offs[:-1], offs[1:]):   # every parameter block
        ref = go[a:b]
        assert np.linalg.norm(g[a:b] - ref) <= 2e-2 * np.linalg.norm(ref) + 1e-7, (a, b)
    np.testing.assert_allclose(P.predict(X), mlp.predict(w, X), rtol=2e-3, atol=2e-4)


def _logged(seeds, tol=1e-6, family="matern"):
    Xs, ys = [], []
    for s in seeds:
        if family == "matern":
            x, A, pxy = problems.matern_cube(3000, seed=s, p=32, p_rad=4)
            symm = "p"
        else:
            x, A, pxy = problems.star(6000, seed=s)
            symm = "n"
        F = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm, rank_log=1))
        X, y = F.rank_log()
        Xs.append(X)
        ys.append(y)
    return np.concatenate(Xs), np.concatenate(ys)


def test_training_on_logged_ranks_fits_unseen_geometries():
    X, y = _logged(range(6))
    Xt, yt = _logged([100, 101])
    P = fb.Predictor(seed=0)
    base = float(np.mean((P.predict(Xt) - yt) ** 2))
    loss = P.train(X, y, epochs=150, batch=128, lr=3e-3)
    test = float(np.mean((P.predict(Xt) - yt) ** 2))
    assert loss < 0.2 * base and test < 0.3 * base, (base, loss, test)


def test_predicted_widths_cut_sketch_rows_at_equal_error():
    # the star curve's boxes have ranks well below their point counts at 1e-6 (the Matern
    # cube at this size is nearly full rank, where no prediction can save rows)
    X, y = _logged(range(8), family="star")
    P = fb.Predictor(seed=0)
    P.train(X, y, epochs=150, batch=128, lr=3e-3)
    x, A, pxy = problems.star(5000, seed=50)
    xo, Ao, po = configs.star(5000, seed=50)
    D = Ao.dense()
    B = np.asfortranarray(np.random.default_rng(0).standard_normal((5000, 2)))
    out = {}
    for name, opts in [("fixed", dict(sketch=1)), ("learned", dict(sketch=1, predictor=P, sketch_p=12))]:
        F = fb.rskelf(A, x, 64, 1e-6, pxy, dict(symm="n", profile=True, **opts))
        prof = F.profile()
        Xs, it, rel = fb.rskelf_ir_sv(F, B, ir_tol=1e-10, max_iter=10)
        r = np.linalg.norm(D @ Xs - B, axis=0) / np.linalg.norm(B, axis=0)
        out[name] = dict(rows_per_sketch=prof["sketch_rows"] / max(prof["n_sketch"], 1), id_rows=prof["id_rows"],
                         sketched=prof["n_sketch"], redo=prof["n_sketch_redo"], err=r.max(), ir=it,
                         t_compress=prof["t_compress"])
    print("fixed vs learned sketch widths:", out)
    assert out["fixed"]["err"] <= 1e-10 and out["learned"]["err"] <= 1e-10
    # the learned widths cut the sketch of a box and the rows the IDs fold in all
    assert out["learned"]["rows_per_sketch"] < 0.8 * out["fixed"]["rows_per_sketch"], out
    assert out["learned"]["id_rows"] < out["fixed"]["id_rows"], out
