"""opts.stop as a predicate stop(levels_done, l) (rskelf.m:128,172), host logic (no GPU)."""
import math

import numpy as np
import pytest

import flam_b200 as fb
from flam_b200 import api


class _FakeTree:
    """hypoct of a 2D problem with 4 levels: box sizes 2, 1, 0.5, 0.25 (root first)."""

    def tree(self):
        l = np.array([[2.0, 1.0, 0.5, 0.25], [2.0, 1.0, 0.5, 0.25]])
        return dict(nlvl=4, l=l)

    def free(self):
        self.freed = True


@pytest.fixture
def fake_tree(monkeypatch):
    seen = {}

    def fake_hypoct(x, occ, lvlmax=math.inf, ext=None):
        seen.update(x=x, occ=occ, lvlmax=lvlmax, ext=ext)
        return _FakeTree()

    monkeypatch.setattr(api, "hypoct", fake_hypoct)
    return seen


def test_predicate_becomes_the_level_count_of_its_first_true(fake_tree):
    x = np.zeros((2, 10))
    calls = []

    def stop(done, l):
        calls.append((done, float(l[0])))
        return done >= 2

    assert api._stop_levels(stop, x, 16, {"lvlmax": 7}) == 2
    # called leaf level first, with the number of levels already done (rskelf.m:172)
    assert calls == [(0, 0.25), (1, 0.5), (2, 1.0)]
    assert fake_tree["occ"] == 16 and fake_tree["lvlmax"] == 7
    # a size rule: stop once boxes are wider than 0.75
    assert api._stop_levels(lambda done, l: l[0] > 0.75, x, 16, {}) == 2
    assert api._stop_levels(lambda done, l: False, x, 16, {}) == math.inf
    assert api._stop_levels(lambda done, l: True, x, 16, None) == 0


def test_rskelf_passes_the_equivalent_count(fake_tree, monkeypatch):
    got = {}

    class Stop(Exception):
        pass

    def fake_c_opts(opts):
        got.update(opts)
        raise Stop

    monkeypatch.setattr(api, "_c_opts", fake_c_opts)
    x, A, pxy = fb.problems.star(500, seed=1)
    with pytest.raises(Stop):
        fb.rskelf(A, x, 64, 1e-10, pxy, dict(symm="n", stop=lambda done, l: done >= 3))
    assert got["stop"] == 3 and got["symm"] == "n"
    with pytest.raises(fb.FlamError) as e:
        fb.rskelf_batched([A], [x], 64, 1e-10, pxy, dict(stop=lambda done, l: done >= 1))
    assert e.value.identifier == "FLAM:rskelf:invalidArg"


def test_level_count_matches_the_oracle_predicate(monkeypatch):
    """On the oracle's own tree, the count equals the levels the oracle's rskelf runs with
    the same predicate."""
    from oracle import configs
    from oracle.rskelf import rskelf as o_rskelf
    from oracle.tree import hypoct as o_hypoct

    class OracleTree:
        def __init__(self, x, occ):
            self.t = o_hypoct(x, occ)

        def tree(self):
            return dict(nlvl=self.t["nlvl"], l=self.t["l"])

        def free(self):
            pass

    monkeypatch.setattr(api, "hypoct", lambda x, occ, lvlmax=math.inf, ext=None: OracleTree(x, occ))
    xo, Ao, po = configs.star(1200, seed=2, clustered=False)
    for stop in (lambda done, l: done >= 2, lambda done, l: l[0] > 0.3):
        n = api._stop_levels(stop, xo, 64, {})
        Fo = o_rskelf(Ao, xo, 64, 1e-8, po, dict(symm="n", stop=stop), order="level_sync")
        assert n == len(Fo["stats"])
