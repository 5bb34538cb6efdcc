"""Seeded synthetic inputs with the shapes of the benchmark workloads.

The reference's datasets (testDiego/, diegoVel/, testSid/, read by main.cpp:62-145) are not
available, so every workload here is drawn from a PCG64 generator with a recorded seed.

Workloads (sizes can be scaled down with ``n=``/``blocks_per_side=`` for tests):

* ``uniform_potential``  -- N = M = 65,536 sources on U[0,1)^2, values U[-1,1]; targets are a
  separate copy of the source coordinates; theta = 0.5.
* ``lamb_oseen_force``   -- N = 1,048,576 sources around a Lamb-Oseen vortex at (0.5, 0.5):
  radius Rayleigh(sigma = 0.1), angle uniform, value exp(-r^2/0.01)/N * (1 + 0.01 N(0,1));
  targets are 32 x 32 MRAG blocks of 32 x 32 points, origins (bx, by)/32, h = 1/1024.
* ``gaussian_mixture_potential`` -- N = M = 4,194,304: 80% from 16 isotropic Gaussians
  (centres U[0.1,0.9]^2, sigma log-uniform in [0.005, 0.05]), 20% U[0,1)^2, clipped to
  [0,1); values U[-1,1]; targets are a copy of the source coordinates.
* ``vortex_sheet_force`` -- N = 16,777,216 sources on x ~ U[0,1),
  y = 0.5 + 0.05 sin(2 pi x) + N(0, 0.002^2), values U[0.5,1.5]/N; targets are 64 x 64 MRAG
  blocks of 32 x 32 points, origins (bx, by)/64, h = 1/2048.

Block ib of an MRAG grid with ``g`` blocks per side has origin (bx/g, by/g) with
ib = bx + g*by.
"""
from __future__ import annotations

import numpy as np

ONE_BELOW = np.nextafter(1.0, 0.0)


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def mrag_grid(blocks_per_side: int, h: float, origin=(0.0, 0.0), extent=1.0):
    g = blocks_per_side
    by, bx = np.divmod(np.arange(g * g), g)
    x0 = origin[0] + bx * (extent / g)
    y0 = origin[1] + by * (extent / g)
    return x0.astype(np.float64), y0.astype(np.float64), np.full(g * g, h, np.float64)


def uniform_potential(n=65536, seed=1451):
    r = _rng(seed)
    xs = r.random(n)
    ys = r.random(n)
    vs = r.uniform(-1.0, 1.0, n)
    return dict(kind="potential", theta=0.5, xs=xs, ys=ys, vs=vs, xt=xs.copy(), yt=ys.copy(),
                seed=seed, name=f"uniform_potential_N{n}")


def lamb_oseen_force(n=1 << 20, blocks_per_side=32, h=None, seed=1452):
    r = _rng(seed)
    rad = r.rayleigh(0.1, n)
    ang = r.uniform(0.0, 2 * np.pi, n)
    xs = 0.5 + rad * np.cos(ang)
    ys = 0.5 + rad * np.sin(ang)
    vs = np.exp(-rad * rad / 0.01) / n * (1.0 + 0.01 * r.standard_normal(n))
    h = 1.0 / (32 * blocks_per_side) if h is None else h
    x0, y0, hs = mrag_grid(blocks_per_side, h)
    return dict(kind="force", theta=0.5, xs=xs, ys=ys, vs=vs, x0s=x0, y0s=y0, hs=hs,
                seed=seed, name=f"lamb_oseen_force_N{n}_B{blocks_per_side ** 2}")


def gaussian_mixture_potential(n=1 << 22, theta=0.5, seed=1453):
    r = _rng(seed)
    ng = int(round(0.8 * n))
    centres = r.uniform(0.1, 0.9, (16, 2))
    sig = np.exp(r.uniform(np.log(0.005), np.log(0.05), 16))
    comp = r.integers(0, 16, ng)
    pts = np.empty((n, 2))
    pts[:ng] = centres[comp] + sig[comp, None] * r.standard_normal((ng, 2))
    pts[ng:] = r.random((n - ng, 2))
    pts = np.clip(pts, 0.0, ONE_BELOW)
    perm = r.permutation(n)
    pts = pts[perm]
    xs = np.ascontiguousarray(pts[:, 0])
    ys = np.ascontiguousarray(pts[:, 1])
    vs = r.uniform(-1.0, 1.0, n)
    return dict(kind="potential", theta=theta, xs=xs, ys=ys, vs=vs, xt=xs.copy(), yt=ys.copy(),
                seed=seed, name=f"gaussian_mixture_potential_N{n}")


def vortex_sheet_force(n=1 << 24, blocks_per_side=64, h=None, seed=1454):
    r = _rng(seed)
    xs = r.random(n)
    ys = 0.5 + 0.05 * np.sin(2 * np.pi * xs) + 0.002 * r.standard_normal(n)
    vs = r.uniform(0.5, 1.5, n) / n
    h = 1.0 / (32 * blocks_per_side) if h is None else h
    x0, y0, hs = mrag_grid(blocks_per_side, h)
    return dict(kind="force", theta=0.5, xs=xs, ys=ys, vs=vs, x0s=x0, y0s=y0, hs=hs,
                seed=seed, name=f"vortex_sheet_force_N{n}_B{blocks_per_side ** 2}")


WORKLOADS = {
    "uniform_potential": uniform_potential,
    "lamb_oseen_force": lamb_oseen_force,
    "gaussian_mixture_potential": gaussian_mixture_potential,
    "vortex_sheet_force": vortex_sheet_force,
}
