"""Reference options handled on the host around the device path (GPU).

* ``symm = 'h'``: no LDL on the device; like the reference under Octave
  (rskelf.m:124-127) the factorization takes LU and warns FLAM:rskelf:octaveLDL.
* ``opts.stop`` as a predicate stop(levels_done, l) (rskelf.m:128,172).
"""
import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import problems
from oracle import configs

pytestmark = pytest.mark.gpu


def test_symm_h_factors_with_lu_and_warns():
    N, tol = 2000, 1e-10
    x, A, pxy = problems.circle(N)
    with pytest.warns(UserWarning, match="FLAM:rskelf:octaveLDL"):
        F = fb.rskelf(A, x, 64, tol, pxy, dict(symm="h"))
    assert F.symm == "n"
    Fn = fb.rskelf(A, x, 64, tol, pxy, dict(symm="n"))
    np.testing.assert_array_equal(F.level_stats(), Fn.level_stats())
    D = configs.circle(N)[1].dense()
    B = np.asfortranarray(np.random.default_rng(6).standard_normal((N, 2)))
    X = fb.rskelf_sv(F, B)
    assert np.linalg.norm(D @ X - B) / np.linalg.norm(B) < 1e3 * tol


def test_stop_predicate_equals_its_level_count():
    from oracle.rskelf import rskelf as o_rskelf
    N = 4000
    x, A, pxy = problems.star(N, seed=3, clustered=False)
    xo, Ao, po = configs.star(N, seed=3, clustered=False)
    Fp = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n", stop=lambda done, l: done >= 2))
    Fc = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n", stop=2))
    np.testing.assert_array_equal(Fp.level_stats(), Fc.level_stats())
    # a size rule: the same levels as the oracle with the same predicate
    rule = lambda done, l: l[0] > 0.2   # noqa: E731
    Fs = fb.rskelf(A, x, 64, 1e-8, pxy, dict(symm="n", stop=rule))
    Fo = o_rskelf(Ao, xo, 64, 1e-8, po, dict(symm="n", stop=rule), order="level_sync")
    rows = np.asarray(Fs.level_stats())
    assert len(rows) == len(Fo["stats"])
    ro = np.asarray([[s["lvl"], s["nblk"], s["nrem1"]] for s in Fo["stats"]])
    np.testing.assert_array_equal(rows[:, :2], ro[:, :2])
    assert np.all(np.abs(rows[:, 2] - ro[:, 2]) <= 0.01 * ro[:, 2] + 2)
