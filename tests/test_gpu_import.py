"""Factorizations given in the reference's F layout, imported and applied on the device.

hifie2/hifie3 produce factorizations in rskelf format and apply them with rskelf_sv/mv
(hifie/hifie_sv.m:21); this checks that an imported F is applied exactly as the
oracle's loops over F.factors apply it: for the oracle's own rskelf factorizations (in
the reference's box order) and for random factor sequences whose consecutive factors
share indices (which must then act one after another).
"""
import numpy as np
import pytest

import flam_b200 as fb
from oracle import configs
from oracle.rskelf import (rskelf as o_rskelf, rskelf_cholmv as o_cholmv, rskelf_cholsv as o_cholsv,
                           rskelf_logdet as o_logdet, rskelf_mv as o_mv, rskelf_sv as o_sv)

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("symm", ["n", "s", "p"])
def test_import_oracle_factorization(symm):
    if symm == "n":
        x, A, pxy = configs.star(2500, seed=2, clustered=False)
    else:
        x, A, pxy = configs.circle(2000)
    Fo = o_rskelf(A, x, 64, 1e-10, pxy, dict(symm=symm), order="reference")
    F = fb.factor_import(Fo)
    N = x.shape[1]
    B = np.asfortranarray(np.random.default_rng(1).standard_normal((N, 3)))
    for trans in ("n", "t", "c"):
        assert rel(fb.rskelf_sv(F, B, trans), o_sv(Fo, B, trans)) < 1e-12
        assert rel(fb.rskelf_mv(F, B, trans), o_mv(Fo, B, trans)) < 1e-12
        if symm == "p":
            assert rel(fb.rskelf_cholmv(F, B, trans), o_cholmv(Fo, B, trans)) < 1e-12
            assert rel(fb.rskelf_cholsv(F, B, trans), o_cholsv(Fo, B, trans)) < 1e-12
    ld, lo = fb.rskelf_logdet(F), o_logdet(Fo)
    assert abs(ld.real - lo.real) <= 1e-12 * max(1.0, abs(lo.real))
    assert abs(np.exp(1j * ld.imag) - np.exp(1j * lo.imag)) < 1e-9   # angles: 0 and 2 pi - eps agree
    # a round trip through the export gives the same factors
    ex = F.factors()["factors"]
    assert len(ex) == len(Fo["factors"])
    for a, b in zip(ex[:50], Fo["factors"][:50]):
        np.testing.assert_array_equal(a["sk"], b["sk"])
        np.testing.assert_array_equal(a["T"], b["T"])


def random_factors(N, nfac, symm, seed):
    rng = np.random.default_rng(seed)
    fs = []
    for _ in range(nfac):
        k, r = int(rng.integers(0, 10)), int(rng.integers(1, 10))
        idx = rng.choice(N, k + r, replace=False)
        sk, rd = idx[:k], idx[k:]
        f = dict(sk=sk, rd=rd, T=0.3 * rng.standard_normal((k, r)), E=0.3 * rng.standard_normal((k, r)))
        if symm == "p":
            Lm = np.tril(0.2 * rng.standard_normal((r, r)), -1) + np.diag(rng.uniform(1.0, 2.0, r))
            f.update(L=Lm, U=None, p=None, F=None)
        else:
            Lm = np.tril(0.3 * rng.standard_normal((r, r)), -1) + np.eye(r)
            Um = np.triu(0.3 * rng.standard_normal((r, r)), 1) + np.diag(rng.uniform(1.0, 2.0, r) *
                                                                      rng.choice([-1.0, 1.0], r))
            f.update(L=Lm, U=Um, p=rng.permutation(r), F=0.3 * rng.standard_normal((r, k)))
        fs.append(f)
    return dict(N=N, symm=symm, factors=fs)


@pytest.mark.parametrize("symm", ["n", "p"])
def test_import_overlapping_sequence(symm):
    # 60 factors on 200 points: consecutive factors often share indices
    Fo = random_factors(200, 60, symm, seed=3 if symm == "n" else 4)
    F = fb.factor_import(Fo)
    assert 1 < F.info()["nstep"] <= 60
    B = np.asfortranarray(np.random.default_rng(2).standard_normal((200, 4)))
    for trans in ("n", "t"):
        assert rel(fb.rskelf_sv(F, B, trans), o_sv(Fo, B, trans)) < 1e-12
        assert rel(fb.rskelf_mv(F, B, trans), o_mv(Fo, B, trans)) < 1e-12
    if symm == "p":
        assert rel(fb.rskelf_cholsv(F, B), o_cholsv(Fo, B)) < 1e-12
