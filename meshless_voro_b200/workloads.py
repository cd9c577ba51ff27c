"""Seeded synthetic generator sets with the shapes of the benchmark configurations.

No public dataset is involved; every set is drawn from numpy's PCG64 with a fixed
seed so tests, the benchmark and the CPU baseline see identical inputs.
"""
from __future__ import annotations

import numpy as np


def perturbed_grid(anchor, width, count, pert, rng):
    """count^3 lattice points (i + 0.5 + pert * U(-0.5, 0.5)) * width / count + anchor,
    clamped to the box -- the recipe of the reference's perturbed_grid test helper
    (voronoi.rs:840-859) with a seeded generator."""
    anchor = np.asarray(anchor, dtype=np.float64)
    width = np.asarray(width, dtype=np.float64)
    n = np.arange(count ** 3)
    idx = np.stack([n // count ** 2, (n % count ** 2) // count, n % count], axis=1).astype(np.float64)
    jit = rng.uniform(-0.5, 0.5, size=idx.shape) if pert != 0 else 0.0
    pos = (idx + 0.5 + pert * jit) * width / count + anchor
    return np.clip(pos, anchor, anchor + width)


def perturbed_plane(anchor, width, count, pert, rng):
    """count^2 points in the z = anchor.z + width.z / 2 plane (voronoi.rs:882-900)."""
    anchor = np.asarray(anchor, dtype=np.float64)
    width = np.asarray(width, dtype=np.float64)
    n = np.arange(count ** 2)
    i, j = (n // count).astype(np.float64), (n % count).astype(np.float64)
    jit = rng.uniform(-0.5, 0.5, size=(count ** 2, 2)) if pert != 0 else np.zeros((count ** 2, 2))
    pos = np.stack([i + 0.5 + pert * jit[:, 0], j + 0.5 + pert * jit[:, 1],
                    np.full(count ** 2, 0.5 * count)], axis=1) * width / count + anchor
    return np.clip(pos, anchor, anchor + width)


def jittered_lattice_32(seed=1):
    """32^3 lattice of spacing 1/32 in [0,1]^3, U(+-0.25 spacing) jitter, rectangular."""
    rng = np.random.default_rng(seed)
    g = perturbed_grid([0, 0, 0], [1, 1, 1], 32, 0.5, rng)
    return dict(generators=g, anchor=np.zeros(3), width=np.ones(3), dimensionality=3,
                periodic=False, name="jittered_lattice_32^3_rect")


def exact_lattice(count=64):
    """count^3 unperturbed lattice (i + 0.5) / count, periodic unit box."""
    g = perturbed_grid([0, 0, 0], [1, 1, 1], count, 0.0, None)
    return dict(generators=g, anchor=np.zeros(3), width=np.ones(3), dimensionality=3,
                periodic=True, name=f"exact_lattice_{count}^3_periodic")


def poisson(n, seed=3, periodic=True, dim=3):
    """n i.i.d. uniform points in the unit box."""
    rng = np.random.default_rng(seed)
    g = rng.uniform(0.0, 1.0, size=(n, 3))
    if dim < 3:
        g[:, dim:] = 0.0
    return dict(generators=g, anchor=np.zeros(3), width=np.ones(3), dimensionality=dim,
                periodic=periodic, name=f"poisson_{n}_{'periodic' if periodic else 'rect'}")


def poisson_256(seed=3):
    """256^3 = 16,777,216 i.i.d. uniform points in [0,1)^3, periodic (the headline)."""
    return poisson(256 ** 3, seed=seed, periodic=True)


def clustered(n=8388608, nclumps=2000, seed=4, periodic=True, dim=3):
    """Clustered, uneven density: half of the n points i.i.d. uniform in [0,1)^dim, half
    drawn from nclumps isotropic Gaussian clumps with centres uniform in the box, sigma
    log-uniform in [1e-4, 1e-2] and Pareto(alpha = 1.5) weights normalised to the clump
    counts (multinomial); clump points are wrapped into the unit box.  With the defaults
    the local density spans about four orders of magnitude."""
    rng = np.random.default_rng(seed)
    nb = n // 2
    pts = [rng.uniform(0.0, 1.0, size=(nb, 3))]
    centres = rng.uniform(0.0, 1.0, size=(nclumps, 3))
    sigma = np.exp(rng.uniform(np.log(1e-4), np.log(1e-2), size=nclumps))
    w = rng.pareto(1.5, size=nclumps) + 1.0
    counts = rng.multinomial(n - nb, w / w.sum())
    for c, s, k in zip(centres, sigma, counts):
        if k:
            pts.append(np.mod(c + s * rng.standard_normal((k, 3)), 1.0))
    g = np.concatenate(pts)
    if dim < 3:
        g[:, dim:] = 0.0
    return dict(generators=g, anchor=np.zeros(3), width=np.ones(3), dimensionality=dim,
                periodic=periodic, name=f"clustered_{n}_{nclumps}clumps_{'periodic' if periodic else 'rect'}")


def batch_jobs(njobs=4096, seed=5, nmin=1000, nmax=200000):
    """An uneven batch of independent tessellations (the batched configuration): per
    job N log-uniform in [nmin, nmax]; 3D with probability 0.8, else 2D; i.i.d. uniform
    points or a jittered lattice (U(+-0.25 spacing), about N points) with probability
    1/2 each; box sides U[0.5, 2] at an anchor U[-1, 1]; periodic with probability 1/2;
    and with probability 0.1 a partial build whose mask leaves out a random 25 % of the
    generators.  Returns the list of job dicts (generators, anchor, width,
    dimensionality, periodic, mask)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(njobs):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        dim = 3 if rng.uniform() < 0.8 else 2
        width = rng.uniform(0.5, 2.0, 3)
        anchor = rng.uniform(-1.0, 1.0, 3)
        periodic = bool(rng.uniform() < 0.5)
        if rng.uniform() < 0.5:
            u = rng.uniform(0.0, 1.0, size=(n, 3))
        else:
            k = max(1, int(round(n ** (1.0 / dim))))
            idx = np.indices((k,) * dim).reshape(dim, -1).T.astype(np.float64)
            u = np.full((idx.shape[0], 3), 0.5)
            u[:, :dim] = (idx + 0.5 + rng.uniform(-0.25, 0.25, size=idx.shape)) / k
        g = anchor + u * width
        if dim == 2:
            g[:, 2] = anchor[2] + 0.5 * width[2]
        mask = rng.uniform(size=len(g)) >= 0.25 if rng.uniform() < 0.1 else None
        jobs.append(dict(generators=g, anchor=anchor, width=width, dimensionality=dim,
                         periodic=periodic, mask=mask))
    return jobs


def grid_example(count=64, pert=0.95, seed=1):
    """The reference's examples/grid_3d.rs input: a count^3 perturbed grid (perturbation
    pert, 0 for the perfect grid) in the non-periodic unit box -- the configuration its
    published CPU times are quoted on."""
    rng = np.random.default_rng(seed)
    g = perturbed_grid([0, 0, 0], [1, 1, 1], count, pert, rng if pert else None)
    kind = "perfect" if pert == 0 else f"perturbed{pert}"
    return dict(generators=g, anchor=np.zeros(3), width=np.ones(3), dimensionality=3,
                periodic=False, name=f"grid_{count}^3_{kind}_rect")
