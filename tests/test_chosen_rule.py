"""The chosen form's per-problem precision rule (host logic, no GPU)."""
from flam_b200 import chosen


def test_rule_picks_refinement_only_for_short_3d_products():
    # 3D Laplace sphere, 64 RHS: the TF32 sketch at 1e-6 plus FP64 refinement
    assert chosen.choose(3, 131072, 64, 1e-10, "n") == "tf32-refine"
    assert chosen.choose(3, 16384, 64, 1e-10, "n") == "tf32-refine"
    # 2D curves: ranks grow like log(1/tol), the FP64 sketch at tol wins
    assert chosen.choose(2, 262144, 256, 1e-10, "n") == "fp64-sketch"
    # long residual products: no refinement
    assert chosen.choose(3, 1 << 20, 64, 1e-10, "n") == "fp64-sketch"
    # SPD covariance: the FP64 sketch
    assert chosen.choose(3, 262144, 4, 1e-10, "p") == "fp64-sketch"
    # loose targets need no refinement
    assert chosen.choose(3, 4096, 4, 1e-5, "n") == "fp64-sketch"


def test_factor_options_of_each_form():
    o = chosen.factor_opts("fp64-sketch", "n")
    assert o["sketch"] == 2 and "predictor" not in o
    o = chosen.factor_opts("tf32-refine", "p", predictor=object(), stream=7, profile=True)
    assert o["sketch"] == 1 and o["sketch_p"] == 12 and o["stream"] == 7 and o["profile"]
    assert chosen.factor_tol("tf32-refine", 1e-10) == chosen.REFINE_FACTOR_TOL
    assert chosen.factor_tol("fp64-sketch", 1e-10) == 1e-10


class _FakeX:
    def __init__(self):
        self.copied = None

    def copy_(self, B):
        self.copied = B


class _FakeF:
    def __init__(self, symm):
        self.symm = symm
        self.solved = False

    def sv_(self, X):
        self.solved = True


def test_spd_failure_of_a_sketched_factorization_falls_back_to_lu(monkeypatch):
    """A sketched 'p' factorization whose redundant block fails Cholesky is redone with
    symm 'n' on the same options; other errors propagate."""
    import numpy as np
    from flam_b200 import _lib, api
    calls = []

    def fake_rskelf(A, x, occ, tol, pxy, opts):
        calls.append(opts["symm"])
        if opts["symm"] == "p":
            raise _lib.FlamError(chosen.NOT_SPD, "FLAM:rskelf:notPosDef: a redundant block is not positive definite")
        return _FakeF(opts["symm"])

    monkeypatch.setattr(api, "rskelf", fake_rskelf)
    x = np.zeros((3, 100))
    B = np.zeros((100, 2))
    X = _FakeX()
    F, form, it, rel = chosen.solve(None, x, 64, None, B, X, 1e-10, "p", form="fp64-sketch")
    assert calls == ["p", "n"] and F.symm == "n" and F.solved and X.copied is B
    assert form == "fp64-sketch" and it == 0 and rel is None

    def failing(A, x, occ, tol, pxy, opts):
        raise _lib.FlamError(1, "FLAM:rskelf:invalidArg: bad")

    monkeypatch.setattr(api, "rskelf", failing)
    import pytest
    with pytest.raises(_lib.FlamError):
        chosen.solve(None, x, 64, None, B, X, 1e-10, "p", form="fp64-sketch")

    def not_spd(A, x, occ, tol, pxy, opts):
        calls.append(opts["symm"])
        raise _lib.FlamError(chosen.NOT_SPD, "FLAM:rskelf:notPosDef: a redundant block is not positive definite")

    monkeypatch.setattr(api, "rskelf", not_spd)
    calls.clear()
    with pytest.raises(_lib.FlamError):   # only symm 'p' is retried, and only once
        chosen.solve(None, x, 64, None, B, X, 1e-10, "n", form="fp64-sketch")
    assert calls == ["n"]
    calls.clear()
    with pytest.raises(_lib.FlamError):
        chosen.solve(None, x, 64, None, B, X, 1e-10, "p", form="fp64-sketch")
    assert calls == ["p", "n"]
