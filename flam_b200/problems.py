"""Seeded synthetic problems on the rskelf path (the reference ships no dataset).

Each generator returns ``(x, A, pxyfun)`` with ``x`` d x N FP64 and registry
descriptors for the matrix and the proxy.  Seeds go through
``numpy.random.default_rng(seed)``.

* ``ie_circle``   the reference README's example: double layer on the unit circle,
                  single-layer ring proxy (rskelf/test/ie_circle.m:33-35,97-115)
* ``circle``      A = I + (2 pi/N) K, K = -log r/(2 pi), points theta_i = 2 pi i/N
* ``star``        r(t) = 1 + a cos(k t) curve, t = 2 pi u with u ~ Beta(1/2,1/2) (clustered)
                  or uniform, arc-length weights w, A = I + K diag(w)
* ``sphere``      Fibonacci sphere + seeded rotation, A = I + (4 pi/N) K, K = 1/(4 pi r)
* ``matern_cube`` uniform points in [0,1]^3, A = K + 1e-2 I, Matern-3/2, length scale 0.1
* ``instance_batch``  N log-uniform in [1024, 16384], a ~ U[0.1,0.4], k ~ U{3..9}
"""
import math

import numpy as np

from .registry import Kernel, Proxy


def ie_circle(N=16384, p=64):
    theta = np.arange(1, N + 1) * 2 * math.pi / N
    x = np.stack([np.cos(theta), np.sin(theta)])
    A = Kernel("laplace2d_dl", scale=2 * math.pi / N, dval=-0.5 * (1 + 1.0 / N), normals=x)
    return x, A, Proxy("ring", p, "laplace2d", scale=2 * math.pi / N)


def circle(N=16384, p=64):
    theta = np.arange(1, N + 1) * 2 * math.pi / N
    x = np.stack([np.cos(theta), np.sin(theta)])
    A = Kernel("laplace2d", scale=2 * math.pi / N, dval=1.0)
    return x, A, Proxy("ring", p, "laplace2d", scale=2 * math.pi / N)


def star_points(N, a, k, theta):
    r = 1.0 + a * np.cos(k * theta)
    dr = -a * k * np.sin(k * theta)
    x = np.stack([r * np.cos(theta), r * np.sin(theta)])
    speed = np.sqrt(r * r + dr * dr)
    gap = (np.roll(theta, -1) - np.roll(theta, 1)) % (2 * math.pi)
    return x, speed * gap / 2.0


def star(N=262144, a=0.3, k=5, seed=0, clustered=True, p=64, symm="n"):
    rng = np.random.default_rng(seed)
    if clustered:
        theta = 2 * math.pi * np.sort(rng.beta(0.5, 0.5, size=N))
    else:
        theta = np.arange(1, N + 1) * 2 * math.pi / N
    x, w = star_points(N, a, k, theta)
    A = Kernel("laplace2d", scale=1.0, dval=1.0, weights=w)
    return x, A, Proxy("ring", p, "laplace2d", scale=1.0, two_sided=(symm == "n"))


def random_rotation(rng):
    G = rng.standard_normal((3, 3))
    Q, R = np.linalg.qr(G)
    Q = Q * np.sign(np.diag(R))[None, :]
    if np.linalg.det(Q) < 0:
        Q[:, 0] = -Q[:, 0]
    return Q


def fibonacci_sphere(p, radius=1.0):
    i = np.arange(p, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / p
    rr = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * math.pi * (3.0 - math.sqrt(5.0))
    return radius * np.stack([rr * np.cos(phi), rr * np.sin(phi), z])


def sphere(N=131072, p=256, seed=0):
    rng = np.random.default_rng(seed)
    x = random_rotation(rng) @ fibonacci_sphere(N, 1.0)
    A = Kernel("laplace3d", scale=4 * math.pi / N, dval=1.0)
    return x, A, Proxy("sphere", p, "laplace3d", scale=4 * math.pi / N)


def matern_cube(N=262144, seed=0, ell=0.1, p=64, p_rad=8):
    rng = np.random.default_rng(seed)
    x = rng.random((3, N))
    A = Kernel("matern32", scale=1.0, dval=1.0 + 1e-2, param=1.0 / ell)
    return x, A, Proxy("annulus", p, "matern32", scale=1.0, param=1.0 / ell, p_rad=p_rad)


def instance_batch(count=4096, seed=0, nmin=1024, nmax=16384):
    rng = np.random.default_rng(seed)
    N = np.round(np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count))).astype(np.int64)
    a = rng.uniform(0.1, 0.4, size=count)
    k = rng.integers(3, 10, size=count)
    return N, a, k


def instance(N, a, k, p=64):
    """One member of the batch: uniform theta on a star curve, arc-length weights."""
    theta = np.arange(1, N + 1) * 2 * math.pi / N
    x, w = star_points(int(N), float(a), int(k), theta)
    A = Kernel("laplace2d", scale=1.0, dval=1.0, weights=w)
    return x, A, Proxy("ring", p, "laplace2d", scale=1.0, two_sided=True)
