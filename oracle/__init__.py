"""CPU oracle for FLAM's recursive skeletonization factorization.

TEST INFRASTRUCTURE ONLY.  This package is a line-by-line NumPy/SciPy
restatement of the reference MATLAB code on the rskelf path:

* ``core/hypoct.m`` and ``core/hypoct_perm.m``   -> :mod:`oracle.tree`
* ``core/id.m``                                   -> :mod:`oracle.idecomp`
* ``rskelf/rskelf.m``, ``rskelf/sv/*.m``,
  ``rskelf/mv/*.m``, ``rskelf_sv.m``, ``rskelf_mv.m`` -> :mod:`oracle.rskelf`
* ``core/snorm.m``                                -> :mod:`oracle.snorm`
* the kernels / proxy functions of the reference's test drivers
  (``rskelf/test/ie_circle.m``, ``ie_cube1.m``, ``cov_circle1.m``,
  ``cov_circle2.m``, ``hifie/test/cov_cube2.m``)  -> :mod:`oracle.registry`

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import it, and only as the checker.  The product path
(``flam_b200``) never imports, links or executes anything in here.

Parity status: the tree (``hypoct``) is pinned against the reference
README's ``ie_circle`` run (levels, boxes per level); the per-level skeleton
counts of that run are reproduced by the ``order="reference"`` mode.  Pivot
sequences of the LAPACK CPQR the reference calls are not pinned by any
reference test (they depend on the BLAS build), so ``sk``/``rd`` parity is
stated against this oracle, not against MATLAB.
"""
