"""flam_id_noalloc: the ID for callers that cannot allocate device memory.

Such a caller (a MEX/oct gateway inside MATLAB or Octave, whose GPU memory
manager owns the device heap; a thread that must not enter cudaMalloc/cudaFree)
passes device buffers for the matrix and the outputs, and the library takes
its scratch from an array compiled into it.  Checked here against flam_id, the
allocating entry point, on two calls in a row.  This file is collected last so
a failure here never hides the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest

import flam_b200 as fb

pytestmark = pytest.mark.gpu


def noalloc_id(A, rank_or_tol, Tmax, rrqr_iter=-1):
    import torch
    L = fb.lib()
    m, n = A.shape
    Ad = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()          # column-major m x n
    k = torch.zeros(1, dtype=torch.int64, device="cuda")
    perm = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    T = torch.full((n * n // 4 + 1,), np.nan, dtype=torch.float64, device="cuda")
    it = torch.zeros(1, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.flam_id_noalloc(C.c_void_p(Ad.data_ptr()), m, n, m, float(rank_or_tol), float(Tmax), int(rrqr_iter),
                           C.c_void_p(k.data_ptr()), C.c_void_p(perm.data_ptr()), C.c_void_p(T.data_ptr()),
                           C.c_void_p(it.data_ptr()), C.c_void_p(stream))
    torch.cuda.synchronize()
    assert rc == 0, L.flam_last_error()
    kk = int(k.item())
    p = perm.cpu().numpy()
    Tm = T[: kk * (n - kk)].cpu().numpy().reshape(n - kk, kk).T if 0 < kk < n else np.zeros((kk, n - kk))
    return p[:kk], p[kk:], Tm, int(it.item())


def test_noalloc_matches_flam_id_on_consecutive_calls():
    rng = np.random.default_rng(11)
    cases = [
        (rng.standard_normal((90, 60)) @ np.diag(0.6 ** np.arange(60)) @ rng.standard_normal((60, 60)), 1e-9, 2.0),
        (rng.standard_normal((300, 128)) @ np.diag(0.8 ** np.arange(128)) @ rng.standard_normal((128, 128)),
         1e-10, 1.05),                                             # n at the limit, RRQR swaps
    ]
    for A, rot, Tmax in cases:
        sk0, rd0, T0, it0 = fb.id(A, rot, Tmax)
        for _ in range(2):                                        # two calls in a row share the array
            sk, rd, T, it = noalloc_id(A, rot, Tmax)
            np.testing.assert_array_equal(sk, sk0)
            np.testing.assert_array_equal(rd, rd0)
            assert it == it0
            np.testing.assert_allclose(T, T0, rtol=1e-12, atol=1e-14)
            if T.size:
                err = np.linalg.norm(A[:, rd] - A[:, sk] @ T, 2) / np.linalg.norm(A, 2)
                assert err < 1e3 * rot


def test_noalloc_rejects_oversize_and_host_pointers():
    import torch
    L = fb.lib()
    n = 129
    A = torch.zeros(10, n, dtype=torch.float64, device="cuda")
    out = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    k = torch.zeros(1, dtype=torch.int64, device="cuda")
    perm = torch.zeros(n, dtype=torch.int64, device="cuda")
    rc = L.flam_id_noalloc(C.c_void_p(A.data_ptr()), 10, n, 10, 1e-6, 2.0, -1, C.c_void_p(k.data_ptr()),
                           C.c_void_p(perm.data_ptr()), C.c_void_p(out.data_ptr()), None, None)
    assert rc == 1 and b"FLAM_ID_NOALLOC_NMAX" in L.flam_last_error()
    host = np.zeros((10, 8))
    rc = L.flam_id_noalloc(C.c_void_p(host.ctypes.data), 10, 8, 10, 1e-6, 2.0, -1, C.c_void_p(k.data_ptr()),
                           C.c_void_p(perm.data_ptr()), C.c_void_p(out.data_ptr()), None, None)
    assert rc == 1 and b"device pointers" in L.flam_last_error()


def test_noalloc_reports_the_rrqr_limit_through_niter():
    """flam_id warns FLAM:id:maxIterCount when the RRQR loop stops at rrqr_iter
    (core/id.m:232-235); the asynchronous no-alloc call reports it as niter == rrqr_iter."""
    rng = np.random.default_rng(5)
    A = rng.standard_normal((300, 128)) @ np.diag(0.8 ** np.arange(128)) @ rng.standard_normal((128, 128))
    with pytest.warns(UserWarning, match="maxIterCount"):
        sk0, rd0, T0, it0 = fb.id(A, 1e-10, 1.05, rrqr_iter=1)
    assert it0 == 1
    for _ in range(2):
        sk, rd, T, it = noalloc_id(A, 1e-10, 1.05, rrqr_iter=1)
        assert it == 1
        np.testing.assert_array_equal(sk, sk0)
        np.testing.assert_array_equal(rd, rd0)
        np.testing.assert_allclose(T, T0, rtol=1e-12, atol=1e-14)


def test_noalloc_empty_matrix():
    """n = 0: k = 0 and niter = 0, as flam_id gives (core/id.m:64-68)."""
    import torch
    L = fb.lib()
    k = torch.full((1,), 7, dtype=torch.int64, device="cuda")
    it = torch.full((1,), 7, dtype=torch.int64, device="cuda")
    rc = L.flam_id_noalloc(None, 5, 0, 5, 1e-6, 2.0, -1, C.c_void_p(k.data_ptr()), None, None,
                           C.c_void_p(it.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0, L.flam_last_error()
    assert int(k.item()) == 0 and int(it.item()) == 0
