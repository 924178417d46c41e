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
