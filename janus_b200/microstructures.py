"""Seeded synthetic microstructures for the benchmark and test problems.

The reference ships no datasets; these generators produce the phase maps
and property fields of the benchmark configurations (all seeded, so a run is
reproducible):

* ``square_inclusion``: the 2D square inclusion (centred, or in the corner
  like sphinx/tutorials/square_basic/square_basic.py:35-37);
* ``random_spheres``: non-overlapping spheres by random sequential addition
  under periodic distance, up to a volume fraction;
* ``ellipses``: 2D random elliptical inclusions with periodic wrap;
* ``ellipsoid``: one centred ellipse / ellipsoid on a cartesian grid of
  given physical size (the generator of notebooks/gen_ellipsoid.py:12-38,
  without its HDF5 output: h5py is not part of this build);
* ``voronoi``: periodic nearest-site partition with a random phase per cell;
* ``gaussian_field``: a stationary Gaussian random field with squared-
  exponential correlation, made by spectral filtering of white noise.
"""
from __future__ import annotations

import math

import numpy as np


def square_inclusion(n, side=None, centered=True, a=0.5):
    """uint8 phase map (1 inside the square).  centered: side `side` (default
    n/2) centred in the cell; otherwise the tutorial's corner square
    [0, ceil(n a - 0.5))^2 (square_basic.py:36-37)."""
    phase = np.zeros((n, n), dtype=np.uint8)
    if centered:
        side = n // 2 if side is None else int(side)
        lo = (n - side) // 2
        phase[lo:lo + side, lo:lo + side] = 1
    else:
        imax = int(np.ceil(n * a - 0.5))
        phase[:imax, :imax] = 1
    return phase


def ellipsoid(radii, size, shape):
    """int8 phase map of a 2D ellipse or 3D ellipsoid centred in a grid.

    ``radii`` (2 or 3 floats) and ``size`` (the grid's side lengths) are in
    the same units of length; ``shape`` is the number of cells per side.
    A cell is 1 when its centre lies inside or on the ellipsoid, else 0
    (notebooks/gen_ellipsoid.py:12-38).  Cell centres along an axis of
    length L and n cells sit at -L(n-1)/(2n) ... L(n-1)/(2n), n evenly
    spaced points."""
    radii, size, shape = tuple(radii), tuple(size), tuple(int(n) for n in shape)
    if not (len(radii) == len(size) == len(shape)) or len(shape) not in (2, 3):
        raise ValueError("radii, size and shape must all have length 2 or 3")
    acc = np.zeros(shape)
    for d, (r, L, n) in enumerate(zip(radii, size, shape)):
        h = 0.5 * L * (n - 1) / n
        c = np.linspace(-h, h, num=n) / r
        view = [1] * len(shape)
        view[d] = n
        acc = acc + (c * c).reshape(view)
    return (acc <= 1).astype(np.int8)


def _periodic_delta(d, n):
    d = np.abs(d)
    return np.minimum(d, n - d)


def random_spheres(n, radius=8, volume_fraction=0.3, seed=0, max_attempts=1_000_000):
    """uint8 phase map of non-overlapping spheres (periodic), placed by random
    sequential addition until the voxel volume fraction reaches the target.
    Centres are uniform in [0, n)^3; two spheres may not have centre distance
    below 2 radius (periodic); a voxel is inside when its centre distance^2 is
    <= radius^2.  Returns (phase, centres)."""
    rng = np.random.default_rng(seed)
    phase = np.zeros((n, n, n), dtype=np.uint8)
    centres = []
    r = int(math.ceil(radius))
    offs = np.arange(-r, r + 1)
    dz, dy, dx = np.meshgrid(offs, offs, offs, indexing="ij")
    target = volume_fraction * n ** 3
    count = 0
    attempts = 0
    while count < target and attempts < max_attempts:
        attempts += 1
        c = rng.uniform(0, n, size=3)
        if centres:
            C = np.asarray(centres)
            d = _periodic_delta(C - c, n)
            if np.any((d * d).sum(axis=1) < (2 * radius) ** 2):
                continue
        centres.append(c)
        base = np.floor(c).astype(int)
        z = base[0] + dz
        y = base[1] + dy
        x = base[2] + dx
        d2 = (z + 0.5 - c[0]) ** 2 + (y + 0.5 - c[1]) ** 2 + (x + 0.5 - c[2]) ** 2
        inside = d2 <= radius * radius
        zi, yi, xi = z[inside] % n, y[inside] % n, x[inside] % n
        new = phase[zi, yi, xi] == 0
        phase[zi, yi, xi] = 1
        count += int(new.sum())
    return phase, np.asarray(centres)


def ellipses(n, count, seed=0, amin=4.0, amax=None):
    """uint8 phase map with `count` ellipses (phase 1..count in drawing
    order; later ones overwrite), semi-axes U[amin, amax] (default n/8),
    orientation U[0, pi), centres uniform, periodic wrap."""
    rng = np.random.default_rng(seed)
    amax = n / 8.0 if amax is None else amax
    phase = np.zeros((n, n), dtype=np.uint8)
    i0, i1 = np.meshgrid(np.arange(n) + 0.5, np.arange(n) + 0.5, indexing="ij")
    for e in range(count):
        a, b = rng.uniform(amin, max(amin, amax), size=2)
        th = rng.uniform(0, np.pi)
        c = rng.uniform(0, n, size=2)
        d0 = i0 - c[0]
        d1 = i1 - c[1]
        d0 -= n * np.round(d0 / n)
        d1 -= n * np.round(d1 / n)
        u = d0 * np.cos(th) + d1 * np.sin(th)
        v = -d0 * np.sin(th) + d1 * np.cos(th)
        phase[(u / a) ** 2 + (v / b) ** 2 <= 1.0] = e + 1
    return phase


def voronoi(n, cells=512, seed=0, nphase=2):
    """uint8 phase map of a periodic Voronoi partition of [0, n)^3 into
    `cells` cells (uniform sites), each cell given a random phase in
    [0, nphase) (fair draw).  Uses scipy's periodic k-d tree."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    sites = rng.uniform(0, n, size=(cells, 3))
    cell_phase = rng.integers(0, nphase, size=cells).astype(np.uint8)
    tree = cKDTree(sites, boxsize=n)
    g = np.arange(n) + 0.5
    phase = np.empty((n, n, n), dtype=np.uint8)
    yy, xx = np.meshgrid(g, g, indexing="ij")
    pts = np.empty((n * n, 3))
    pts[:, 1] = yy.ravel()
    pts[:, 2] = xx.ravel()
    for i in range(n):
        pts[:, 0] = g[i]
        _, idx = tree.query(pts)
        phase[i] = cell_phase[idx].reshape(n, n)
    return phase


def gaussian_field(n, dim=3, corr_len=8.0, std=1.5, seed=0):
    """Zero-mean Gaussian random field on an n^dim periodic grid with
    squared-exponential covariance exp(-r^2 / (2 corr_len^2)), built by
    filtering white noise in Fourier space, then standardised to the given
    standard deviation."""
    rng = np.random.default_rng(seed)
    shape = (n,) * dim
    w = rng.standard_normal(shape)
    k = [2 * np.pi * np.fft.fftfreq(n)] * (dim - 1) + [2 * np.pi * np.fft.rfftfreq(n)]
    K = np.meshgrid(*k, indexing="ij", sparse=True)
    k2 = sum(kk * kk for kk in K)
    # amplitude = sqrt of the spectral density of the SE covariance
    amp = np.exp(-0.25 * corr_len ** 2 * k2)
    g = np.fft.irfftn(np.fft.rfftn(w) * amp, s=shape, axes=tuple(range(dim)))
    g -= g.mean()
    g *= std / g.std()
    return g


BATCH_2D_SIZES = (64, 96, 128, 192, 256, 384, 512, 768, 1024)


def batch_2d_problems(count=64, seed=0, sizes=BATCH_2D_SIZES):
    """Seeded batch of two-phase 2D cells of uneven sizes: each draws its
    grid n from ``sizes``, 2-20 ellipses (semi-axes U[4, n/8], uniform
    orientation and centres, periodic wrap) of one inclusion phase, an
    inclusion/matrix shear contrast log-uniform in [10, 1000] (matrix
    mu = 1), Poisson ratios U[0.15, 0.4] per phase, and the reference medium
    at the midpoints of the phases' shear and (plane-strain) bulk moduli:
    mu0 = (mu_min + mu_max)/2, k0 = (k_min + k_max)/2, nu0 = (k0 - mu0)/(2 k0)
    (isotropic.pyx:32-46).  The basic scheme converges only if k0 exceeds
    k_max/2; nu0 = the matrix's nu can violate that when the inclusion's nu
    is the larger one.  Returns a list of dicts with keys n, phase (uint8 0/1
    map), mu, nu (per phase), mu0, nu0."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(sizes))
        k = int(rng.integers(2, 21))
        sub = int(rng.integers(0, 2 ** 31 - 1))
        phase = (ellipses(n, k, seed=sub) > 0).astype(np.uint8)
        contrast = float(np.exp(rng.uniform(np.log(10.0), np.log(1000.0))))
        nu = rng.uniform(0.15, 0.4, size=2)
        mu = np.array([1.0, contrast])
        k = mu / (1.0 - 2.0 * nu)
        mu0 = 0.5 * (mu.min() + mu.max())
        k0 = 0.5 * (k.min() + k.max())
        out.append({"n": n, "phase": phase, "mu": mu, "nu": nu, "mu0": mu0,
                    "nu0": float((k0 - mu0) / (2.0 * k0))})
    return out
