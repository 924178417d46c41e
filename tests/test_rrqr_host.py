"""The device RRQR refinement (flam_b200/csrc/rrqr.cuh), compiled for the host,
against the oracle's restatement of id.m:117-236 on identical (R, p, k) input:
both branches (tolerance mode, and fixed rank with an R22 block)."""
import ctypes as C
import math
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from oracle.idecomp import _id_qr, _id_rrqr

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def rrqr_lib():
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    d = tempfile.mkdtemp()
    so = os.path.join(d, "librrqr_host.so")
    subprocess.check_call([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-o", so,
                           os.path.join(HERE, "native", "rrqr_host.cpp")])
    L = C.CDLL(so)
    L.flam_test_rrqr.restype = C.c_int
    L.flam_test_rrqr.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_double,
                                 C.c_double, C.c_longlong, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return L


def run_host(L, R, p, k, tol, n, Tmax, it=-1):
    rows = R.shape[0]
    Rm = np.zeros((n, n), order="F")
    Rm[:rows, :] = R
    jp = p.astype(np.int32).copy()
    aux = np.zeros(32 * n)
    ni, cap = C.c_int(), C.c_int()
    kk = L.flam_test_rrqr(Rm.ctypes.data, n, n, k, rows, jp.ctypes.data, tol, Tmax, it, aux.ctypes.data,
                          C.byref(ni), C.byref(cap))
    return jp[:kk], jp[kk:], Rm[:kk, kk:].copy(), ni.value


@pytest.mark.parametrize("rot,Tmax", [(1e-8, 1.01), (1e-10, 1.2), (12.0, 1.01), (8.0, 1.05), (1e-6, 2.0)])
def test_rrqr_host_matches_oracle(rrqr_lib, rot, Tmax):
    rng = np.random.default_rng(int(rot * 1e3) % 97 + int(Tmax * 100))
    iters = 0
    for _ in range(25):
        m, n = int(rng.integers(20, 60)), int(rng.integers(10, 40))
        A = rng.standard_normal((m, n)) @ np.diag(0.3 ** np.arange(n)) @ rng.standard_normal((n, n))
        st = _id_qr(A, rot, Tmax)
        _, R, p, k, tol, nn = st
        sk0, rd0, T0, it0 = _id_rrqr(R.copy(), p.copy(), k, tol, nn, Tmax, math.inf)
        sk1, rd1, T1, it1 = run_host(rrqr_lib, R.copy(), p.copy(), k, tol, nn, Tmax)
        iters += it0
        assert it1 == it0
        np.testing.assert_array_equal(sk1, sk0)
        np.testing.assert_array_equal(rd1, rd0)
        np.testing.assert_allclose(T1, T0, rtol=1e-8, atol=1e-10)
    if Tmax < 2:
        assert iters > 0
