"""Seeded synthetic problem generators (oracle side).

The reference publishes no dataset; every configuration is generated from a
seed with ``numpy.random.default_rng(seed)``.  The same generators exist on
the product side (``flam_b200.problems``) and are checked equal by the tests.

* ``ie_circle``  the reference README's worked example (rskelf/test/ie_circle.m:33-35,84-115):
                 double-layer matrix, single-layer ring proxy.
* ``circle``     N points theta_i = 2 pi i / N on the unit circle, A = I + (2 pi/N) K,
                 K = -log r / (2 pi), 64-point ring proxy, occ 64.
* ``star``       theta = 2 pi u, u ~ Beta(0.5, 0.5) sorted (or uniform), curve
                 r(theta) = 1 + a cos(k theta), arc-length weights, A = I + K diag(w).
* ``sphere``     Fibonacci sphere + seeded random rotation, A = I + (4 pi/N) K, K = 1/(4 pi r).
* ``matern_cube`` uniform points in [0,1]^3, A = K + 1e-2 I, Matern-3/2, length scale 0.1.
"""
import math

import numpy as np

from .registry import Kernel, Proxy, fibonacci_sphere


def ie_circle(N=16384, p=64):
    theta = np.arange(1, N + 1) * 2 * math.pi / N
    x = np.stack([np.cos(theta), np.sin(theta)])
    A = Kernel("laplace2d_dl", x, scale=2 * math.pi / N, dval=-0.5 * (1 + 1.0 / N), normals=x)
    pxy = Proxy("ring", 2, p, "laplace2d", scale=2 * math.pi / N)
    return x, A, pxy


def circle(N=16384, p=64):
    theta = np.arange(1, N + 1) * 2 * math.pi / N
    x = np.stack([np.cos(theta), np.sin(theta)])
    A = Kernel("laplace2d", x, scale=2 * math.pi / N, dval=1.0)
    pxy = Proxy("ring", 2, p, "laplace2d", scale=2 * math.pi / N)
    return x, A, pxy


def star_points(N, a, k, theta):
    r = 1.0 + a * np.cos(k * theta)
    dr = -a * k * np.sin(k * theta)
    x = np.stack([r * np.cos(theta), r * np.sin(theta)])
    speed = np.sqrt(r * r + dr * dr)
    tp = np.roll(theta, -1)
    tm = np.roll(theta, 1)
    gap = (tp - tm) % (2 * math.pi)
    w = speed * gap / 2.0
    return x, w


def star(N=262144, a=0.3, k=5, seed=0, clustered=True, p=64, symm="n"):
    rng = np.random.default_rng(seed)
    if clustered:
        u = np.sort(rng.beta(0.5, 0.5, size=N))
        theta = 2 * math.pi * u
    else:
        theta = np.arange(1, N + 1) * 2 * math.pi / N
    x, w = star_points(N, a, k, theta)
    A = Kernel("laplace2d", x, scale=1.0, dval=1.0, weights=w)
    pxy = Proxy("ring", 2, p, "laplace2d", scale=1.0, weights=w, wbar=A.wbar, two_sided=(symm == "n"))
    return x, A, pxy


def random_rotation(rng):
    G = rng.standard_normal((3, 3))
    Q, R = np.linalg.qr(G)
    Q = Q * np.sign(np.diag(R))[None, :]
    if np.linalg.det(Q) < 0:
        Q[:, 0] = -Q[:, 0]
    return Q


def sphere(N=131072, p=256, seed=0):
    rng = np.random.default_rng(seed)
    x = random_rotation(rng) @ fibonacci_sphere(N, 1.0)
    A = Kernel("laplace3d", x, scale=4 * math.pi / N, dval=1.0)
    pxy = Proxy("sphere", 3, p, "laplace3d", scale=4 * math.pi / N)
    return x, A, pxy


def matern_cube(N=262144, seed=0, ell=0.1, p=64, p_rad=8):
    rng = np.random.default_rng(seed)
    x = rng.random((3, N))
    A = Kernel("matern32", x, scale=1.0, dval=1.0 + 1e-2, param=1.0 / ell)
    pxy = Proxy("annulus", 3, p, "matern32", scale=1.0, param=1.0 / ell, p_rad=p_rad)
    return x, A, pxy


def instance_batch(count=4096, seed=0, nmin=1024, nmax=16384):
    """Parameters of the many-instance batch: N log-uniform, a ~ U[0.1,0.4], k ~ U{3..9}."""
    rng = np.random.default_rng(seed)
    N = np.round(np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=count))).astype(np.int64)
    a = rng.uniform(0.1, 0.4, size=count)
    k = rng.integers(3, 10, size=count)
    return N, a, k
