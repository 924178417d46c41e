"""The survey's larger configurations on the device, with their FP64 error from the
on-the-fly FP64 matvec (a dense LU is infeasible at these sizes):

* config 2 at its stated size -- N = 131072 points on a randomly rotated Fibonacci sphere,
  A = I + (4 pi/N) K with the 3D Laplace kernel, 256-point proxy sphere, 64 RHS -- in the
  chosen form (sketched factorization at 1e-6 with learned widths, FP64 refinement to
  1e-10);
* the many-instance pipeline of config 4 (star curves, N log-uniform in [1024, 16384],
  4 RHS) on 256 instances in one batched factorization: every instance's relative
  residual, plain FP64 at 1e-10 and the chosen form.
"""
import os

import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(os.path.dirname(fb.__file__), "predictor_weights.npz")


def test_config2_full_size_chosen_form():
    import torch
    N = 131072
    x, A, pxy = problems.sphere(N, p=256, seed=0)
    xd = torch.from_numpy(np.ascontiguousarray(x.T)).cuda().t()
    P = fb.Predictor.load(WEIGHTS)
    F = fb.rskelf(A, xd, 64, 1e-6, pxy, dict(symm="n", sketch=1, predictor=P, sketch_p=12))
    B = torch.randn(N, 64, dtype=torch.float64, device="cuda").t().contiguous().t()
    X = torch.empty_like(B)
    _, it, rel = F.ir_sv_(B, X, 1e-10, 10)
    R = torch.empty_like(B)
    F.matvec_(X, R, B)
    r = (R.norm(dim=0) / B.norm(dim=0)).max().item()
    print(f"config 2 (N={N}) chosen form: {it} refinement steps, FP64 relative residual {r:.2e}")
    assert r <= 1e-10 and it <= 3


@pytest.mark.parametrize("form", ["plain", "chosen"])
def test_config4_batch_per_instance_error(form):
    import torch
    count = 256
    Ns, a_, k_ = problems.instance_batch(count, seed=3)
    xs, ws = [], []
    for N, a, k in zip(Ns, a_, k_):
        x, A, pxy = problems.instance(N, a, k)
        xs.append(x)
        ws.append(A.weights)
    X = torch.from_numpy(np.ascontiguousarray(np.concatenate(xs, axis=1).T)).cuda().t()
    W = torch.from_numpy(np.concatenate(ws)).cuda()
    off = np.concatenate([[0], np.cumsum(Ns)])
    As = [fb.Kernel("laplace2d", scale=1.0, dval=1.0, weights=W[off[i]:off[i + 1]]) for i in range(count)]
    Ntot = int(off[-1])
    B = torch.randn(Ntot, 4, dtype=torch.float64, device="cuda").t().contiguous().t()
    Xs = torch.empty_like(B)
    if form == "plain":
        F = fb.rskelf_batched(As, X, 64, 1e-10, pxy, dict(symm="n"), sizes=Ns)
        Xs.copy_(B)
        F.sv_(Xs)
    else:
        P = fb.Predictor.load(WEIGHTS)
        F = fb.rskelf_batched(As, X, 64, 1e-6, pxy, dict(symm="n", sketch=1, predictor=P, sketch_p=12), sizes=Ns)
        F.ir_sv_(B, Xs, 1e-10, 10)
    R = torch.empty_like(B)
    F.matvec_(Xs, R, B)
    seg = torch.from_numpy(np.repeat(np.arange(count), Ns)).cuda()
    rn = torch.zeros(count, 4, dtype=torch.float64, device="cuda").index_add_(0, seg, R * R)
    bn = torch.zeros(count, 4, dtype=torch.float64, device="cuda").index_add_(0, seg, B * B)
    err = (rn / bn).sqrt().max(dim=1).values
    print(f"config 4 ({count} instances, {Ntot} points) {form}: per-instance residual max {err.max().item():.2e}")
    assert err.max().item() <= 1e-10
