"""Seeded synthetic point sets shaped like the workloads the reference is
used on (uniform, clustered, boundary-curve, degenerate)."""
import numpy as np


def uniform(n, seed):
    return np.random.default_rng(seed).random((2, n))


def blobs(n, seed, nblob=8, sigma=0.01):
    rng = np.random.default_rng(seed)
    c = rng.random((2, nblob))
    k = rng.integers(0, nblob, n)
    p = c[:, k] + sigma * rng.standard_normal((2, n))
    return p


def starfish(n, seed, arms=5, amp=0.3):
    """Points equispaced in angle on r = 1 + amp cos(arms t), with outward
    unit normals."""
    t = 2 * np.pi * np.arange(n) / n
    r = 1 + amp * np.cos(arms * t)
    dr = -amp * arms * np.sin(arms * t)
    x = np.stack([r * np.cos(t), r * np.sin(t)])
    tan = np.stack([dr * np.cos(t) - r * np.sin(t), dr * np.sin(t) + r * np.cos(t)])
    nrm = np.stack([tan[1], -tan[0]])
    nrm /= np.linalg.norm(nrm, axis=0)
    return x, nrm


def near_curve_targets(n, seed, arms=5, amp=0.3):
    rng = np.random.default_rng(seed)
    t = rng.random(n) * 2 * np.pi
    r = 1 + amp * np.cos(arms * t)
    dr = -amp * arms * np.sin(arms * t)
    x = np.stack([r * np.cos(t), r * np.sin(t)])
    tan = np.stack([dr * np.cos(t) - r * np.sin(t), dr * np.sin(t) + r * np.cos(t)])
    nrm = np.stack([tan[1], -tan[0]])
    nrm /= np.linalg.norm(nrm, axis=0)
    d = 10.0 ** rng.uniform(-3, -1, n) * rng.choice([-1.0, 1.0], n)
    return x + d * nrm


def grid_lines(m):
    """A lattice whose coordinates sit exactly on box center lines."""
    g = np.arange(m + 1) / m
    x, y = np.meshgrid(g, g)
    return np.stack([x.ravel(), y.ravel()])


def with_duplicates(n, seed, ndup):
    p = uniform(n, seed)
    p[:, :ndup] = np.array([[0.3], [0.7]])
    return p


def complex_normal(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
