"""Kernel and proxy registry (oracle side).

The reference passes ``A`` and ``pxyfun`` as MATLAB function handles; the
concrete handles on the rskelf path live in its test drivers.  The registry
restates them as data:

* ``laplace2d``     -K = log(r)/(2 pi) single layer      rskelf/test/ie_circle.m:85-95 ('s')
* ``laplace2d_dl``  double layer (r.n_y)/(2 pi r^2)      rskelf/test/ie_circle.m:91-94 ('d')
* ``laplace3d``     1/(4 pi r)                             rskelf/test/ie_cube1.m:115-121
* ``gaussian``      exp(-0.5 (scale r)^2)                  rskelf/test/cov_circle1.m:130-136
* ``matern32``      (1 + sqrt3 scale r) exp(-sqrt3 scale r) rskelf/test/cov_circle2.m:129-135

A matrix entry is ``A(i,j) = s * w_j * K(x_i, x_j)`` for ``i != j`` and
``A(i,i) = dval`` (the reference's ``A(I == J) = ...`` diagonal replacement,
ie_circle.m:98-103, or ``K(0) + nugget``, cov_circle1.m:139-144).

Proxies (the reference's ``pxyfun_``):

* ``ring``    p points ``1.5 (cos t, sin t)``, t = 2 pi (1..p)/p, scaled by the
              box size and shifted to its centre; ellipse filter
              ``sum(((x-ctr)./l).^2) < 1.5^2``                ie_circle.m:35,106-115
* ``sphere``  p Fibonacci points on the radius-1.5 sphere; ellipsoid filter
              (the reference draws a random subset of an icosphere, ie_cube1.m:31-32)
* ``annulus`` base ring/shell scaled to max|.| = 1, p_rad radii in
              [0, 3/scale], shifted by ``1.5*base.*l + ctr``; box filter
              ``max(|x-ctr|./l) < 1.5``                       cov_circle1.m:34-40,146-152

For non-uniform column weights with ``symm='n'`` the proxy block is
``[s K(pxy,slf) diag(w_slf); s wbar K(pxy,slf)]``: the first half spans the
outgoing far field ``A(far,slf)``, the second the incoming one
``A(slf,far)' = s diag(w_far) K(far,slf)``; one interpolation matrix must
serve both.
"""
import math

import numpy as np

KERNELS = ("laplace2d", "laplace2d_dl", "laplace3d", "gaussian", "matern32")
KERNEL_ID = {k: i for i, k in enumerate(KERNELS)}
PROXIES = ("ring", "sphere", "annulus")
PROXY_ID = {k: i for i, k in enumerate(PROXIES)}


def kfun(kind, xt, ys, param=1.0, normals=None):
    """Kernel block K(xt, ys): xt d x m targets, ys d x n sources -> m x n."""
    diff = xt[:, :, None] - ys[:, None, :]
    r2 = np.sum(diff * diff, axis=0)
    if kind == "laplace2d":
        return -1.0 / (2 * math.pi) * np.log(np.sqrt(r2))
    if kind == "laplace2d_dl":
        rdotn = diff[0] * normals[0][None, :] + diff[1] * normals[1][None, :]
        return 1.0 / (2 * math.pi) * rdotn / r2
    if kind == "laplace3d":
        return 1.0 / (4 * math.pi) / np.sqrt(r2)
    if kind == "gaussian":
        dr = param * np.sqrt(r2)
        return np.exp(-0.5 * dr * dr)
    if kind == "matern32":
        dr = param * np.sqrt(r2)
        return (1.0 + math.sqrt(3.0) * dr) * np.exp(-math.sqrt(3.0) * dr)
    raise ValueError(f"unknown kernel {kind}")


class Kernel:
    """Matrix ``A(I,J)`` from the registry (replaces the reference's ``Afun``)."""

    def __init__(self, kind, x, scale=1.0, dval=1.0, param=1.0, weights=None, normals=None):
        if kind not in KERNELS:
            raise ValueError(f"FLAM:gpu:unsupportedKernel: {kind}")
        self.kind = kind
        self.x = np.asarray(x, dtype=np.float64)
        self.scale = float(scale)
        self.dval = float(dval)
        self.param = float(param)
        self.weights = None if weights is None else np.asarray(weights, dtype=np.float64)
        self.normals = None if normals is None else np.asarray(normals, dtype=np.float64)
        self.wbar = 1.0 if self.weights is None else float(np.mean(self.weights))

    def __call__(self, I, J):
        I = np.asarray(I, dtype=np.int64)
        J = np.asarray(J, dtype=np.int64)
        if I.size == 0 or J.size == 0:
            return np.zeros((I.size, J.size))
        nrm = None if self.normals is None else self.normals[:, J]
        with np.errstate(divide="ignore", invalid="ignore"):
            A = self.scale * kfun(self.kind, self.x[:, I], self.x[:, J], self.param, nrm)
        if self.weights is not None:
            A = A * self.weights[J][None, :]
        eq = I[:, None] == J[None, :]
        A[eq] = self.dval
        return A

    def dense(self):
        n = self.x.shape[1]
        return self(np.arange(n), np.arange(n))


def fibonacci_sphere(p, radius=1.0):
    i = np.arange(p, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / p
    rr = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * math.pi * (3.0 - math.sqrt(5.0))
    return radius * np.stack([rr * np.cos(phi), rr * np.sin(phi), z])


class Proxy:
    """Proxy function from the registry (replaces the reference's ``pxyfun``)."""

    def __init__(self, kind, d, p, kernel_kind, scale=1.0, param=1.0, p_rad=None, two_sided=False, wbar=1.0,
                 weights=None):
        if kind not in PROXIES:
            raise ValueError(f"FLAM:gpu:unsupportedProxy: {kind}")
        self.kind = kind
        self.d = d
        self.p = p
        self.kernel_kind = kernel_kind
        self.scale = float(scale)
        self.param = float(param)
        self.two_sided = bool(two_sided)
        self.wbar = float(wbar)
        self.weights = weights
        self.p_rad = p_rad
        if kind == "ring":
            assert d == 2
            t = np.arange(1, p + 1) * 2 * math.pi / p
            self.pts = 1.5 * np.stack([np.cos(t), np.sin(t)])
            self.shift = None
        elif kind == "sphere":
            assert d == 3
            self.pts = fibonacci_sphere(p, 1.5)
            self.shift = None
        else:
            if d == 2:
                t = np.arange(1, p + 1) * 2 * math.pi / p
                base = np.stack([np.cos(t), np.sin(t)])
            else:
                base = fibonacci_sphere(p, 1.0)
            base = base / np.max(np.abs(base), axis=0)
            nrad = p_rad if p_rad is not None else (p if d == 2 else int(round(p ** 0.5)))
            self.p_rad = nrad
            R = 3.0 / param
            radii = np.linspace(0.0, R, nrad)
            # proxy(:, i, j) = base(:, i) * radii(j), flattened column-major (cov_circle1.m:38)
            self.pts = (base[:, :, None] * radii[None, None, :]).reshape(d, -1, order="F")
            self.shift = np.repeat(1.5 * base[:, :, None], nrad, axis=2).reshape(d, -1, order="F")

    def npxy(self):
        n = self.pts.shape[1]
        return 2 * n if self.two_sided else n

    def points(self, l, ctr):
        if self.shift is None:
            return self.pts * l[:, None] + ctr[:, None]
        return self.pts + self.shift * l[:, None] + ctr[:, None]

    def keep(self, x, nbr, l, ctr):
        if len(nbr) == 0:
            return np.zeros(0, dtype=bool)
        y = (x[:, nbr] - ctr[:, None]) / l[:, None]
        if self.kind in ("ring", "sphere"):
            return np.sum(y * y, axis=0) < 1.5 ** 2
        return np.max(np.abs(y), axis=0) < 1.5

    def __call__(self, x, slf, nbr, l, ctr):
        """[Kpxy, nbr] = pxyfun(x, slf, nbr, l, ctr)."""
        pxy = self.points(l, ctr)
        with np.errstate(divide="ignore", invalid="ignore"):
            K = self.scale * kfun(self.kernel_kind, pxy, x[:, slf], self.param)
        if self.weights is not None:
            Kw = K * self.weights[slf][None, :]
            K = np.concatenate([Kw, self.wbar * K], axis=0) if self.two_sided else Kw
        nbr = np.asarray(nbr, dtype=np.int64)
        return K, nbr[self.keep(x, nbr, l, ctr)]
