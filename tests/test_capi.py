"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and rejects bad arguments with the reference's identifiers
before touching the device."""
import os
import re

import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "flam.h")).read()
    return sorted(set(re.findall(r"FLAM_API\s+[\w\s\*]+?\b(flam_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = fb.lib()
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.EXPORTS)
    assert b"sm_100a" in L.flam_version()


def test_build_recipe_targets_sm100a_only():
    """Every translation unit and the link use one -gencode: sm_100a code, no PTX for other arches."""
    from flam_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert set(build.SOURCES) == {f for f in os.listdir(build.CSRC) if f.endswith(".cu")}


def test_bad_arguments_fail_before_the_device():
    x, A, pxy = fb.problems.star(500, seed=1)
    cases = [
        (dict(symm="q"), "FLAM:chksymm:invalidSymm"),
        (dict(Tmax=0.5), "FLAM:id:invalidTmax"),
    ]
    for opts, ident in cases:
        with pytest.raises(fb.FlamError) as e:
            fb.rskelf(A, x, 64, 1e-10, pxy, opts)
        assert e.value.identifier == ident
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf(A, x, -1, 1e-10, pxy)
    assert e.value.identifier == "FLAM:hypoct:invalidOcc"
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf(A, x, 64, -1.0, pxy)
    assert e.value.identifier == "FLAM:id:invalidRankOrTol"
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf(lambda i, j: np.zeros((len(i), len(j))), x, 64, 1e-10, pxy)
    assert e.value.identifier == "FLAM:gpu:unsupportedHandle"
    with pytest.raises(fb.FlamError) as e:
        fb.Kernel("helmholtz")
    assert e.value.identifier == "FLAM:gpu:unsupportedKernel"
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf(A, x, 64, 1e-10, fb.Proxy("sphere", 64))
    assert e.value.identifier == "FLAM:gpu:invalidProxy"


def test_generators_match_oracle():
    from oracle import configs
    for a, b in [(fb.problems.star(3000, seed=2), configs.star(3000, seed=2)),
                 (fb.problems.circle(1000), configs.circle(1000)),
                 (fb.problems.sphere(2000, seed=1), configs.sphere(2000, seed=1)),
                 (fb.problems.matern_cube(1000, seed=3), configs.matern_cube(1000, seed=3)),
                 (fb.problems.ie_circle(512), configs.ie_circle(512))]:
        np.testing.assert_array_equal(a[0], b[0])
        if a[1].weights is not None:
            np.testing.assert_array_equal(a[1].weights, b[1].weights)
        assert a[1].scale == b[1].scale and a[1].dval == b[1].dval
    Na, aa, ka = fb.problems.instance_batch(64, seed=3)
    Nb, ab, kb = configs.instance_batch(64, seed=3)
    np.testing.assert_array_equal(Na, Nb)
    np.testing.assert_array_equal(ka, kb)


def test_factor_import_rejects_bad_factors():
    good = dict(sk=np.array([0]), rd=np.array([1]), T=np.ones((1, 1)), L=np.ones((1, 1)), U=np.ones((1, 1)),
                p=np.array([0]), E=np.ones((1, 1)), F=np.ones((1, 1)))
    for bad, ident in [(dict(rd=np.array([5])), "FLAM:gpu:invalidFactor"),
                       (dict(rd=np.array([0])), "FLAM:gpu:invalidFactor"),
                       (dict(p=np.array([3])), "FLAM:gpu:invalidFactor")]:
        f = dict(good, **bad)
        with pytest.raises(fb.FlamError) as e:
            fb.factor_import(dict(N=3, symm="n", factors=[f]))
        assert e.value.identifier == ident
    with pytest.raises(fb.FlamError) as e:
        fb.factor_import(dict(N=3, symm="q", factors=[good]))
    assert e.value.identifier == "FLAM:chksymm:invalidSymm"
