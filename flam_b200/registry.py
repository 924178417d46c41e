"""Kernel and proxy registry: the device-side replacement of the reference's
function handles ``A(I,J)`` and ``pxyfun(x,slf,nbr,l,ctr)`` (rskelf/rskelf.m:35-53).

A matrix entry is ``A(i,j) = scale * w_j * K(x_i, x_j)`` for ``i != j`` and
``A(i,i) = dval``; the kernels and proxies are those of the reference's test
drivers:

=============  ===============================================  =====================================
kind           K(x, y)                                          reference
=============  ===============================================  =====================================
laplace2d      -log|x-y| / (2 pi)                               rskelf/test/ie_circle.m:85-95
laplace2d_dl   ((x-y).n_y) / (2 pi |x-y|^2)                      rskelf/test/ie_circle.m:91-94
laplace3d      1 / (4 pi |x-y|)                                 rskelf/test/ie_cube1.m:115-121
gaussian       exp(-(param |x-y|)^2 / 2)                        rskelf/test/cov_circle1.m:130-136
matern32       (1 + sqrt3 param r) exp(-sqrt3 param r)          rskelf/test/cov_circle2.m:129-135
=============  ===============================================  =====================================

Proxies: ``ring`` (ie_circle.m:35,106-115), ``sphere`` (ie_cube1.m:131-140,
Fibonacci points instead of a random icosphere subset), ``annulus``
(cov_circle1.m:34-40,146-152).
"""
import numpy as np

from . import _lib

KERNELS = {"laplace2d": 0, "laplace2d_dl": 1, "laplace3d": 2, "gaussian": 3, "matern32": 4}
PROXIES = {"none": 0, "ring": 1, "sphere": 2, "annulus": 3}


def _array(a, fortran=False):
    """Keep CUDA tensors as they are (device pointers); make host data float64 NumPy."""
    if type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False):
        return a
    return np.asfortranarray(a, dtype=np.float64) if fortran else np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a):
    if a is None:
        return None
    return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data


class Kernel:
    """Registry matrix; stands where the reference takes the handle ``A``."""

    def __init__(self, kind, scale=1.0, dval=1.0, param=1.0, weights=None, normals=None):
        if kind not in KERNELS:
            raise _lib.FlamError(1, f"FLAM:gpu:unsupportedKernel: {kind!r} is not a registry kernel")
        self.kind = kind
        self.scale = float(scale)
        self.dval = float(dval)
        self.param = float(param)
        self.weights = None if weights is None else _array(weights)
        self.normals = None if normals is None else _array(normals, fortran=True)

    def c_struct(self):
        return _lib.FlamKernel(KERNELS[self.kind], self.scale, self.dval, self.param, _ptr(self.weights),
                               _ptr(self.normals))


class Proxy:
    """Registry proxy; stands where the reference takes ``pxyfun``."""

    def __init__(self, kind, p, kernel="laplace2d", scale=1.0, param=1.0, p_rad=1, two_sided=False):
        if kind not in PROXIES:
            raise _lib.FlamError(1, f"FLAM:gpu:unsupportedProxy: {kind!r} is not a registry proxy")
        self.kind = kind
        self.p = int(p)
        self.kernel = kernel
        self.scale = float(scale)
        self.param = float(param)
        self.p_rad = int(p_rad)
        self.two_sided = bool(two_sided)

    def c_struct(self):
        return _lib.FlamProxy(PROXIES[self.kind], self.p, self.p_rad, KERNELS[self.kernel], self.scale, self.param,
                              1 if self.two_sided else 0)
