"""Seeded synthetic universes for the benchmark and the tests.

The reference reads universes from CSV (src/common_lib/InputOutput/src/
InputOutput.cpp:18-52) and ships a galaxy generator in SI units
(scripts/galaxy-generator.py:143-223).  These generators produce the same
kind of input in code units (G = 1) with every choice pinned here:

* exponential_disc: one central body at the origin at rest, holding
  ``central_ratio`` times the disc-body mass; disc bodies of mass 1/(n-1)
  (so the disc weighs 1) with radii drawn from an exponential distribution of
  scale ``scale`` truncated at ``rmax`` (inverse CDF), uniform azimuths,
  counter-clockwise circular speed for the enclosed mass with Plummer
  softening ``eps``, v_c^2 = G M(<r) r^2 / (r^2 + eps^2)^1.5, and Gaussian
  dispersion of ``dispersion`` x v_c added to each velocity component.
* colliding_discs: two such discs of n/2 bodies at x = -offset and +offset,
  moving at +rel_vel/2 and -rel_vel/2 along y.
* plummer_disc: equal masses 1/n, projected-Plummer radii R = a sqrt(u/(1-u)),
  uniform azimuths, isotropic Gaussian velocities of dispersion ``sigma``.
* ensemble: per-universe seeds, sizes log-uniform in [nmin, nmax], scale
  lengths uniform in [0.5, 2], central-mass ratios log-uniform in [1e3, 1e6].
* jittered_grid: side x side equal masses 1/n on a square lattice of width
  ``size``, each moved by up to +-jitter/2 lattice spacings, Gaussian
  velocities of dispersion ``sigma``.  Its tree is shallow and even, so the
  reference's GPU walk stays inside its 32-entry stack
  (src/Simulation/src/BarnesHutCuda.cu:400) at 262,144 bodies, unlike the
  discs.

Arrays come back as (mass[n], pos[n, 2], vel[n, 2]) float64, C-contiguous,
matching the Bodies host layout (interleaved x, y).
"""
from __future__ import annotations

import numpy as np

Universe = tuple[np.ndarray, np.ndarray, np.ndarray]


def exponential_disc(n: int, seed: int, *, scale: float = 1.0, rmax: float = 10.0,
                     central_ratio: float = 1e5, dispersion: float = 0.05, G: float = 1.0,
                     eps: float = 0.01) -> Universe:
    if n < 2:
        raise ValueError("a disc needs the central body and at least one disc body")
    rng = np.random.default_rng(seed)
    nd = n - 1
    m_disc = 1.0 / nd
    u = rng.random(nd)
    r = -scale * np.log1p(-u * (1.0 - np.exp(-rmax / scale)))
    phi = rng.random(nd) * (2.0 * np.pi)
    noise = rng.standard_normal((nd, 2))
    order = np.argsort(r, kind="stable")
    enclosed = np.empty(nd)
    enclosed[order] = central_ratio * m_disc + m_disc * np.arange(nd)
    vc = np.sqrt(G * enclosed * r * r / (r * r + eps * eps) ** 1.5)
    c, s = np.cos(phi), np.sin(phi)
    mass = np.empty(n)
    pos = np.zeros((n, 2))
    vel = np.zeros((n, 2))
    mass[0] = central_ratio * m_disc
    mass[1:] = m_disc
    pos[1:, 0] = r * c
    pos[1:, 1] = r * s
    vel[1:, 0] = -vc * s + dispersion * vc * noise[:, 0]
    vel[1:, 1] = vc * c + dispersion * vc * noise[:, 1]
    return mass, pos, vel


def colliding_discs(n: int, seed: int, *, offset: float = 20.0, rel_vel: float = 0.5,
                    **disc) -> Universe:
    if n < 4 or n % 2:
        raise ValueError("colliding_discs needs an even n >= 4")
    parts = []
    for k, (dx, dvy) in enumerate(((-offset, 0.5 * rel_vel), (offset, -0.5 * rel_vel))):
        m, p, v = exponential_disc(n // 2, seed * 2 + k, **disc)
        p[:, 0] += dx
        v[:, 1] += dvy
        parts.append((m, p, v))
    return tuple(np.ascontiguousarray(np.concatenate(x)) for x in zip(*parts))  # type: ignore


def plummer_disc(n: int, seed: int, *, a: float = 1.0, sigma: float = 0.3,
                 umax: float = 1.0 - 1e-6) -> Universe:
    rng = np.random.default_rng(seed)
    u = rng.random(n) * umax
    r = a * np.sqrt(u / (1.0 - u))
    phi = rng.random(n) * (2.0 * np.pi)
    vel = rng.standard_normal((n, 2)) * sigma
    pos = np.stack([r * np.cos(phi), r * np.sin(phi)], axis=1)
    mass = np.full(n, 1.0 / n)
    return mass, np.ascontiguousarray(pos), np.ascontiguousarray(vel)


def jittered_grid(side: int, seed: int, *, jitter: float = 0.5, size: float = 10.0,
                  sigma: float = 0.01) -> Universe:
    rng = np.random.default_rng(seed)
    ij = np.stack(np.meshgrid(np.arange(side), np.arange(side), indexing="ij"), -1).reshape(-1, 2)
    pos = (ij + 0.5 + (rng.random(ij.shape) - 0.5) * jitter) * (size / side)
    n = pos.shape[0]
    vel = rng.standard_normal((n, 2)) * sigma
    return np.full(n, 1.0 / n), np.ascontiguousarray(pos), np.ascontiguousarray(vel)


def ensemble_sizes(count: int, seed: int, nmin: int = 1024, nmax: int = 262144) -> np.ndarray:
    rng = np.random.default_rng([seed, 0])
    return np.exp(rng.uniform(np.log(nmin), np.log(nmax), count)).astype(np.int64)


def ensemble(count: int, seed: int, nmin: int = 1024, nmax: int = 262144) -> list[Universe]:
    sizes = ensemble_sizes(count, seed, nmin, nmax)
    rng = np.random.default_rng([seed, 1])
    scales = rng.uniform(0.5, 2.0, count)
    ratios = np.exp(rng.uniform(np.log(1e3), np.log(1e6), count))
    return [exponential_disc(int(sizes[k]), seed * 100003 + k, scale=float(scales[k]),
                             central_ratio=float(ratios[k]))
            for k in range(count)]


def ensemble_batch(count: int, seed: int, nmin: int = 1024, nmax: int = 262144):
    """The ensemble concatenated in universe order, as nb_batch_create takes it:
    (mass[N], pos[N, 2], vel[N, 2], counts[count] uint64)."""
    unis = ensemble(count, seed, nmin, nmax)
    counts = np.array([u[0].shape[0] for u in unis], dtype=np.uint64)
    m, p, v = (np.ascontiguousarray(np.concatenate(x)) for x in zip(*unis))
    return m, p, v, counts


# The five workloads of the benchmark description, by name.
WORKLOADS = {
    "disc16k": dict(n=16384, kind="disc", theta=0.5, steps=1000),
    "collision4m": dict(n=4194304, kind="collision", theta=0.5, steps=100),
    "plummer16m": dict(n=16777216, kind="plummer", theta=0.5, steps=50),
    "collision4m_theta1": dict(n=4194304, kind="collision", theta=1.0, steps=100),
}


def make(kind: str, n: int, seed: int = 0) -> Universe:
    if kind == "disc":
        return exponential_disc(n, seed)
    if kind == "collision":
        return colliding_discs(n, seed)
    if kind == "plummer":
        return plummer_disc(n, seed)
    if kind == "grid":
        side = int(round(np.sqrt(n)))
        if side * side != n:
            raise ValueError("a jittered grid needs a square body count")
        return jittered_grid(side, seed)
    raise ValueError(f"unknown universe kind {kind!r}")
