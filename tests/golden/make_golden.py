"""Generate the golden fixtures of tests/golden from the oracle.

    python tests/golden/make_golden.py

The oracle (oracle/) restates the reference's MATLAB code; these fixtures pin
its outputs on small seeded problems so the device tests compare against fixed
vectors.  The reference publishes no golden vectors of its own; the one
known-answer run it prints (README.md, ie_circle N=16384) is checked directly
in tests/test_oracle.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import configs  # noqa: E402
from oracle.idecomp import id_  # noqa: E402
from oracle.rskelf import rskelf, rskelf_mv, rskelf_sv  # noqa: E402
from oracle.tree import hypoct, hypoct_perm, tree_arrays  # noqa: E402


def save_tree(name, x, occ, **kw):
    t = hypoct(x, occ, **kw)
    a = tree_arrays(t)
    np.savez_compressed(os.path.join(HERE, name), x=x, occ=occ, perm=hypoct_perm(t), **{k: np.asarray(v) for k, v in a.items()},
                        lvlmax=kw.get("lvlmax", np.inf))


def id_cases():
    rng = np.random.default_rng(0)
    out = {}
    for c in range(6):
        m, n = [(40, 30), (200, 20), (15, 30), (40, 30), (64, 64), (300, 50)][c]
        A = rng.standard_normal((m, n)) @ np.diag(0.3 ** np.arange(n)) @ rng.standard_normal((n, n))
        rot, Tmax = [(1e-8, 1.01), (1e-10, 2.0), (1e-6, 2.0), (12.0, 1.01), (1e-12, 2.0), (1e-9, 1.05)][c]
        sk, rd, T, it = id_(A, rot, Tmax)
        out[f"A{c}"] = A
        out[f"p{c}"] = np.array([rot, Tmax])
        out[f"sk{c}"] = sk
        out[f"rd{c}"] = rd
        out[f"T{c}"] = T
        out[f"it{c}"] = it
    np.savez_compressed(os.path.join(HERE, "id_cases.npz"), **out)


def factor_case(name, gen, occ, tol, symm, nrhs=3, seed=11):
    x, A, pxy = gen()
    F = rskelf(A, x, occ, tol, pxy, dict(symm=symm), order="level_sync")
    rng = np.random.default_rng(seed)
    B = rng.standard_normal((x.shape[1], nrhs))
    X = rskelf_sv(F, B)
    Y = rskelf_mv(F, B)
    fs = F["factors"]
    k = np.array([len(f["sk"]) for f in fs])
    r = np.array([len(f["rd"]) for f in fs])
    sk = np.concatenate([np.sort(f["sk"]) for f in fs])
    rows = np.array([[s["lvl"], s["nblk"], s["nrem1"], s["nrem2"]] for s in F["stats"]])
    np.savez_compressed(os.path.join(HERE, name), x=x, B=B, X=X, Y=Y, k=k, r=r, sk_sorted=sk, lvp=F["lvp"],
                        stats=rows, tol=tol, occ=occ, symm=symm)


if __name__ == "__main__":
    rng = np.random.default_rng(1)
    save_tree("tree_star3000.npz", configs.star(3000, seed=3)[0], 32)
    save_tree("tree_cube2000.npz", rng.random((3, 2000)), 16)
    save_tree("tree_sphere4000_lvlmax3.npz", configs.sphere(4000, seed=2)[0], 20, lvlmax=3)
    id_cases()
    factor_case("rskelf_star2048_n.npz", lambda: configs.star(2048, seed=7, clustered=False), 64, 1e-10, "n")
    factor_case("rskelf_circle2048_p.npz", lambda: configs.circle(2048), 64, 1e-10, "p")
    print("ok")
