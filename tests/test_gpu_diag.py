"""rskelf_diag / rskelf_spdiag on the device: diag(F) and diag(inv(F)).

Against the oracle's unfolding (rskelf_diag.m) run on the device's own exported
factors -- rounding only -- and against the dense FP64 matrix: diag(F) ~ diag(A) and
diag(inv(F)) ~ diag(inv(A)) within the factorization tolerance.
"""
import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs
from oracle.rskelf import rskelf_diag as o_diag

pytestmark = pytest.mark.gpu


def oracle_view(F, inst=0):
    d = F.factors(inst)
    return dict(N=d["N"], lvp=d["lvp"], factors=d["factors"], symm=d["symm"])


@pytest.mark.parametrize("symm", ["n", "s", "p"])
def test_diag_matches_oracle_and_dense(symm):
    N, tol = 2500, 1e-10
    if symm == "n":
        x, A, pxy = problems.star(N, seed=8, clustered=False)
        Ad = configs.star(N, seed=8, clustered=False)[1].dense()
    else:
        x, A, pxy = problems.circle(N)
        Ad = configs.circle(N)[1].dense()
    F = fb.rskelf(A, x, 64, tol, pxy, dict(symm=symm))
    Fo = oracle_view(F)
    for dinv in (0, 1):
        D = fb.rskelf_diag(F, dinv)
        Do = o_diag(Fo, dinv)
        assert np.abs(D - Do).max() <= 1e-12 * np.abs(Do).max(), dinv
        np.testing.assert_array_equal(fb.rskelf_spdiag(F, dinv), D)
    assert np.abs(fb.rskelf_diag(F, 0) - np.diag(Ad)).max() <= 1e3 * tol * np.abs(np.diag(Ad)).max()
    Di = np.diag(np.linalg.inv(Ad))
    assert np.abs(fb.rskelf_diag(F, 1) - Di).max() <= 1e3 * tol * np.abs(Di).max()


def test_diag_large_boxes_and_device_output():
    # 3D surface: boxes with n > 128 (global-memory unfolding blocks) at the top levels
    import torch
    x, A, pxy = problems.sphere(4000, p=256, seed=3)
    F = fb.rskelf(A, x, 64, 1e-8, pxy)
    Do = o_diag(oracle_view(F), 1)
    D = torch.zeros(4000, dtype=torch.float64, device="cuda")
    rc = fb.lib().flam_rskelf_diag(F.handle, 1, D.data_ptr())
    assert rc == 0
    assert np.abs(D.cpu().numpy() - Do).max() <= 1e-12 * np.abs(Do).max()


def test_diag_batched_and_errors():
    Ns, aa, kk = problems.instance_batch(3, seed=5, nmin=800, nmax=2000)
    items = [problems.instance(int(n), a, k) for n, a, k in zip(Ns, aa, kk)]
    Fb = fb.rskelf_batched([it[1] for it in items], [it[0] for it in items], 64, 1e-10, items[0][2])
    Db = fb.rskelf_diag(Fb, 1)
    off = 0
    for i, (x, A, pxy) in enumerate(items):
        n = x.shape[1]
        Do = o_diag(oracle_view(Fb, i), 1)
        assert np.abs(Db[off:off + n] - Do).max() <= 1e-12 * np.abs(Do).max()
        off += n
    x, A, pxy = items[0]
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf_diag(fb.rskelf(A, x, 64, 1e-10, pxy, dict(stop=2)))
    assert e.value.identifier == "FLAM:rskelf_diag:partial"
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf_diag(fb.factor_import(oracle_view(Fb, 0)))
    assert e.value.identifier == "FLAM:rskelf_diag:noTree"
