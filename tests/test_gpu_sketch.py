"""Sketched (mixed-precision) compression: the ID of a row sketch Y = Omega K formed in
FP32 on the tensor cores (tcgen05 kind::tf32), FP64 pivoted QR / rank / R11 \\ R12 on Y
(core/id.m:102-114 applied to Y), the posterior check that redoes a box exactly, and FP64
iterative refinement back to the FP64 tolerance."""
import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs

pytestmark = pytest.mark.gpu


def _ranks(F):
    fac = F.factors()["factors"]
    return np.array([len(f["sk"]) for f in fac]), np.array([len(f["rd"]) for f in fac])


@pytest.mark.parametrize("case", ["star", "sphere", "matern"])
def test_sketched_factorization_matches_exact_ranks_and_tolerance(case):
    if case == "star":
        (x, A, pxy), (xo, Ao, po), symm = problems.star(6000, seed=5), configs.star(6000, seed=5), "n"
    elif case == "sphere":
        (x, A, pxy), (xo, Ao, po), symm = (problems.sphere(5000, p=128, seed=1), configs.sphere(5000, p=128, seed=1),
                                           "n")
    else:
        (x, A, pxy), (xo, Ao, po), symm = (problems.matern_cube(4000, seed=2, p=32, p_rad=4),
                                           configs.matern_cube(4000, seed=2, p=32, p_rad=4), "p")
    tol = 1e-6
    Fe = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm))
    Fs = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm, sketch=1, profile=True))
    prof = Fs.profile()
    assert prof["n_sketch"] > 0 and prof["n_sketch_redo"] == 0
    ke, re_ = _ranks(Fe)
    ks, rs = _ranks(Fs)
    # same tree, same boxes per step; ranks of the sketched ID within a few of the exact ID's
    assert Fe.info()["nstep"] == Fs.info()["nstep"]
    assert abs(int(ks.sum()) - int(ke.sum())) <= 0.05 * ke.sum() + 5
    N = x.shape[1]
    D = Ao.dense()
    B = np.asfortranarray(np.random.default_rng(1).standard_normal((N, 2)))
    for F in (Fe, Fs):
        X = fb.rskelf_sv(F, B)
        assert np.linalg.norm(D @ X - B) / np.linalg.norm(B) < 1e3 * tol
    X, it, rel = fb.rskelf_ir_sv(Fs, B, ir_tol=1e-10, max_iter=10)
    r = np.linalg.norm(D @ X - B, axis=0) / np.linalg.norm(B, axis=0)
    assert r.max() <= 1e-10 and rel.max() <= 1e-10


def test_posterior_check_redoes_boxes_whose_rank_fills_the_sketch():
    x, A, pxy = problems.star(5000, seed=3)
    xo, Ao, po = configs.star(5000, seed=3)
    tol = 1e-6
    Fe = fb.rskelf(A, x, 64, tol, pxy, dict(symm="n"))
    # w = n - 40 rows: boxes of rank above w - 2 must go back to the exact ID
    Fs = fb.rskelf(A, x, 64, tol, pxy, dict(symm="n", sketch=1, sketch_p=-40, sketch_guard=2, profile=True))
    prof = Fs.profile()
    assert prof["n_sketch_redo"] > 0
    ke, _ = _ranks(Fe)
    ks, _ = _ranks(Fs)
    assert abs(int(ks.sum()) - int(ke.sum())) <= 0.05 * ke.sum() + 5
    D = Ao.dense()
    B = np.asfortranarray(np.random.default_rng(2).standard_normal((5000, 2)))
    X = fb.rskelf_sv(Fs, B)
    assert np.linalg.norm(D @ X - B) / np.linalg.norm(B) < 1e3 * tol


def test_sketch_off_is_the_exact_path():
    x, A, pxy = problems.star(3000, seed=4)
    F0 = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n", profile=True))
    assert F0.profile()["n_sketch"] == 0


def test_sketched_wide_boxes_and_grid_elimination_reach_fp64_tolerance():
    """A 3D sphere whose top boxes hold more than 1024 points (the wide pivoted QR of the
    sketch) and whose root block takes the grid-wide elimination; the FP64 residual is
    measured by the on-the-fly matvec."""
    import torch
    N = 16384
    x, A, pxy = problems.sphere(N, p=256, seed=7)
    F = fb.rskelf(A, x, 64, 1e-6, pxy, dict(symm="n", sketch=1, profile=True))
    assert F.profile()["n_sketch"] > 0
    nmax = max(len(f["sk"]) + len(f["rd"]) for f in F.factors()["factors"])
    assert nmax > 1024
    B = torch.randn(N, 4, dtype=torch.float64, device="cuda").t().contiguous().t()
    X = torch.empty_like(B)
    _, it, rel = F.ir_sv_(B, X, 1e-10, 10)
    R = torch.empty_like(B)
    F.matvec_(X, R, B)
    r = (R.norm(dim=0) / B.norm(dim=0)).max().item()
    assert r <= 1e-10 and rel.max() <= 1e-10 and it >= 1


def test_autotune_records_a_setting_that_later_factorizations_use():
    x, A, pxy = problems.star(20000, seed=9)
    before = fb.tune_get(2, "laplace2d", 20000)
    best = fb.autotune(A, x, 64, 1e-10, pxy, dict(symm="n"), reps=1)
    assert fb.tune_get(2, "laplace2d", 20000) == best
    assert best["split_ctas"] in (74, 148, 296) and best["split_max"] in (2, 4, 8, 16)
    # the tuned shapes change launch geometry, not the factorization's ranks
    xo, Ao, po = configs.star(20000, seed=9)
    F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="n"))
    fb.tune_set(2, "laplace2d", 20000, before)
    G = fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="n"))
    sf, sg = F.level_stats(), G.level_stats()
    assert np.array_equal(sf[:, :3], sg[:, :3]) or sf.shape == sg.shape
    assert np.all(np.abs(sf[:, 3] - sg[:, 3]) <= 0.002 * sg[:, 3] + 1)
    with pytest.raises(fb.FlamError, match="tune:invalidArg"):
        fb.tune_set(2, "laplace2d", 20000, dict(split_ctas=0, split_max=8, split_min_n=32, tc_smem_max=0))


def test_low_sketch_widths_on_wide_boxes_take_a_second_full_sketch():
    """A box of more than 1024 points whose rank fills its sketch is sketched again at full
    width (the adaptive fallback) instead of taking the exact per-column ID."""
    import time
    import torch
    N = 16384
    x, A, pxy = problems.sphere(N, p=256, seed=11)
    t0 = time.time()
    F = fb.rskelf(A, x, 64, 1e-6, pxy, dict(symm="n", sketch=1, sketch_p=-700, profile=True))
    torch.cuda.synchronize()
    dt = time.time() - t0
    prof = F.profile()
    assert prof["n_sketch_redo"] > 0
    assert dt < 20.0, dt
    B = torch.randn(N, 2, dtype=torch.float64, device="cuda").t().contiguous().t()
    X = torch.empty_like(B)
    _, it, rel = F.ir_sv_(B, X, 1e-10, 10)
    R = torch.empty_like(B)
    F.matvec_(X, R, B)
    assert (R.norm(dim=0) / B.norm(dim=0)).max().item() <= 1e-10


def test_repeated_applies_replay_a_cuda_graph():
    import torch
    x, A, pxy = problems.star(8000, seed=12)
    xo, Ao, po = configs.star(8000, seed=12)
    F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="n"))
    B = torch.randn(8000, 40, dtype=torch.float64, device="cuda").t().contiguous().t()
    X = torch.empty_like(B)
    outs = []
    for _ in range(4):                      # eager, capture + replay, replay, replay
        X.copy_(B)
        F.sv_(X)
        outs.append(X.clone())
    assert F.profile()["graph_replays"] == 3
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
    D = Ao.dense()
    r = np.linalg.norm(D @ outs[-1].cpu().numpy() - B.cpu().numpy()) / np.linalg.norm(B.cpu().numpy())
    assert r < 1e-8
    Y = B.clone()
    F.mv_(Y)                                # another key: eager again
    assert F.profile()["graph_replays"] == 3


def test_two_host_threads_factor_on_one_device():
    """Handles made concurrently from two host threads on one device (per-device kernel
    attributes and per-stream workspaces) give the same factorizations as one thread."""
    import threading
    import torch
    probs = [problems.star(6000, seed=20), problems.sphere(4000, p=128, seed=21)]
    ref = [fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n")).level_stats() for x, A, pxy in probs]
    out = [None, None]
    errs = []

    def work(i):
        try:
            st = torch.cuda.Stream()
            x, A, pxy = probs[i]
            F = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n", stream=st.cuda_stream))
            out[i] = F.level_stats()
        except Exception as e:   # noqa: BLE001 - reported below
            errs.append(e)

    th = [threading.Thread(target=work, args=(i,)) for i in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs, errs
    for a, b in zip(out, ref):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("case", ["star", "sphere", "matern"])
def test_fp64_sketch_meets_tight_tolerance_without_refinement(case):
    """opts.sketch = 2: K's entries and the products in FP64 (FP64 tensor path), so the ID
    of the sketch meets tol 1e-10 directly; ranks within a few of the exact ID's."""
    if case == "star":
        (x, A, pxy), (xo, Ao, po), symm = problems.star(6000, seed=7), configs.star(6000, seed=7), "n"
    elif case == "sphere":
        (x, A, pxy), (xo, Ao, po), symm = (problems.sphere(5000, p=128, seed=3), configs.sphere(5000, p=128, seed=3),
                                           "n")
    else:
        (x, A, pxy), (xo, Ao, po), symm = (problems.matern_cube(4000, seed=4, p=32, p_rad=4),
                                           configs.matern_cube(4000, seed=4, p=32, p_rad=4), "p")
    tol = 1e-10
    Fe = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm))
    Fs = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm, sketch=2, profile=True))
    prof = Fs.profile()
    assert prof["n_sketch"] > 0
    assert prof["sketch_rows"] < prof["sketch_rows_k"]
    ke, _ = _ranks(Fe)
    ks, _ = _ranks(Fs)
    assert Fe.info()["nstep"] == Fs.info()["nstep"]
    assert abs(int(ks.sum()) - int(ke.sum())) <= 0.05 * ke.sum() + 5
    N = x.shape[1]
    D = Ao.dense()
    B = np.asfortranarray(np.random.default_rng(2).standard_normal((N, 3)))
    res = []
    for F in (Fe, Fs):
        X = fb.rskelf_sv(F, B)
        res.append((np.linalg.norm(D @ X - B, axis=0) / np.linalg.norm(B, axis=0)).max())
    # the exact ID's residual is tol times the conditioning (Matern with a 1e-2 nugget: ~1e4);
    # the sketched ID's is within a small factor of it.  A randomized range finder's error is
    # bounded by (1 + sqrt(k/(p-1))) s_{k+1} + (e sqrt(k+p)/p) ||s_{k+1:}||_2 (Halko, Martinsson
    # and Tropp 2011, Thm. 10.6): the second term is the tail's whole energy.  The log kernel
    # on a curve and the Laplace kernel on a sphere have geometrically decaying tails (that
    # norm is ~ s_{k+1}); the Matern covariance in a volume has a flat one (~ sqrt(n - k)
    # s_{k+1}, n - k ~ 100 on this tree), so its factor is allowed to be ten times larger.
    fac = 100 if case == "matern" else 10
    assert res[0] <= (1e-10 if case != "matern" else 1e-8)
    assert res[1] <= max(1e-10, fac * res[0]), res


def test_fp64_sketch_with_predicted_widths_and_invalid_option():
    x, A, pxy = problems.star(12000, seed=8)
    xo, Ao, po = configs.star(12000, seed=8)
    import os
    pred = fb.Predictor.load(os.path.join(os.path.dirname(fb.__file__), "predictor_weights.npz"))
    F = fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="n", sketch=2, predictor=pred, profile=True))
    prof = F.profile()
    assert prof["n_sketch"] > 0
    B = np.asfortranarray(np.random.default_rng(3).standard_normal((12000, 2)))
    X = fb.rskelf_sv(F, B)
    D = Ao.dense()
    assert (np.linalg.norm(D @ X - B, axis=0) / np.linalg.norm(B, axis=0)).max() <= 1e-10
    with pytest.raises(fb.FlamError, match="invalidSketch"):
        fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="n", sketch=3))
