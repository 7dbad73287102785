"""Seeded synthetic kriging workloads.

No public dataset is involved: each workload is generated from a fixed seed
with numpy's ``default_rng`` and has the shape, density, value distribution
and covariance model of one benchmark configuration of the engine:

* ``ok_small``   100x100x50, 2000 conditioning cells, N(0,1) + 0.01*x,
                 spherical (10,10,5), nugget 0.1, k=12                 (seed 1)
* ``sk_ok_large`` 256x256x128 (8.4M cells), 1% conditioning cells,
                 lognormal(0, 0.5), exponential (30,15,6) azimuth 30,
                 nugget 0.05, k=32                                     (seed 2)
* ``indicator``  200x200x100, 1.5% conditioning, 5 categories from
                 thresholding a smooth Gaussian field at the cumulative
                 marginals (0.40, 0.65, 0.80, 0.92); per-category spherical
                 models, k=24                                          (seed 3)
* ``gauss_cv``   200x200x50, 4000 conditioning cells from a Gaussian field with
                 ranges (18,18,6); Gaussian model, nugget 0.05, k=24   (seed 4)
* ``clustered``  512x512x64 (16.8M cells), 0.2% conditioning in 50 Gaussian
                 clusters (sigma 8 cells); Gaussian (40,40,8), nugget 1e-3,
                 k=64 (ill-conditioned)                                 (seed 5)

Arrays are flat in Fortran order (x fastest: node = x + nx*y + nx*ny*z),
undefined cells hold -99 and mask 0. ``scale`` < 1 shrinks every grid axis
(and the conditioning count with the volume) for quick tests while keeping
densities and models.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Tuple

import numpy as np

UNDEFINED = -99.0

SPHERICAL, EXPONENTIAL, GAUSSIAN = 0, 1, 2


@dataclasses.dataclass
class CovSpec:
    cov_type: int
    ranges: Tuple[float, float, float]
    angles: Tuple[float, float, float]
    sill: float
    nugget: float


@dataclasses.dataclass
class Workload:
    name: str
    dims: Tuple[int, int, int]
    data: np.ndarray                 # float32 (continuous) or uint8 (categories)
    mask: np.ndarray                 # uint8
    cov: CovSpec
    radiuses: Tuple[int, int, int]
    max_neighbours: int
    # indicator workloads only
    categories: int = 0
    marginals: Optional[List[float]] = None
    cat_covs: Optional[List[CovSpec]] = None
    cat_radiuses: Optional[List[Tuple[int, int, int]]] = None

    @property
    def n_cells(self) -> int:
        return int(self.dims[0]) * int(self.dims[1]) * int(self.dims[2])


def _scaled_dims(dims, scale):
    return tuple(max(4, int(round(d * scale))) for d in dims)


def _coords(idx, dims):
    nx, ny, _ = dims
    return idx % nx, (idx // nx) % ny, idx // (nx * ny)


def gaussian_field(dims, ranges, rng) -> np.ndarray:
    """Unit-variance stationary field with covariance ~ exp(-3 (h/a)^2).

    White noise convolved (by FFT) with an anisotropic Gaussian kernel
    exp(-x^2 / (2 s^2)), s = a / sqrt(12) per axis; returned flat, Fortran order.
    """
    nx, ny, nz = dims
    noise = rng.standard_normal((nx, ny, nz))
    kern = np.ones((nx, ny, nz))
    for ax, (n, a) in enumerate(zip(dims, ranges)):
        s = max(a / np.sqrt(12.0), 1e-6)
        d = np.minimum(np.arange(n), n - np.arange(n)).astype(np.float64)
        g = np.exp(-d * d / (2 * s * s))
        shape = [1, 1, 1]
        shape[ax] = n
        kern = kern * g.reshape(shape)
    f = np.real(np.fft.ifftn(np.fft.fftn(noise) * np.fft.fftn(kern)))
    f = (f - f.mean()) / f.std()
    return f.reshape(-1, order="F")


def _finish(data_defined, idx, n):
    data = np.full(n, UNDEFINED, dtype=np.float32)
    mask = np.zeros(n, dtype=np.uint8)
    data[idx] = data_defined.astype(np.float32)
    mask[idx] = 1
    return data, mask


def ok_small(scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(1)
    dims = _scaled_dims((100, 100, 50), scale)
    n = dims[0] * dims[1] * dims[2]
    m = max(1, int(round(2000 * n / 500000)))
    idx = rng.choice(n, m, replace=False)
    x, _, _ = _coords(idx, dims)
    vals = rng.standard_normal(m).astype(np.float32) + np.float32(0.01) * x.astype(np.float32)
    data, mask = _finish(vals, idx, n)
    return Workload("ok_small", dims, data, mask,
                    CovSpec(SPHERICAL, (10.0, 10.0, 5.0), (0.0, 0.0, 0.0), 1.0, 0.1),
                    (10, 10, 5), 12)


def sk_ok_large(scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(2)
    dims = _scaled_dims((256, 256, 128), scale)
    n = dims[0] * dims[1] * dims[2]
    m = max(1, int(n * 0.01))
    idx = rng.choice(n, m, replace=False)
    vals = rng.lognormal(0.0, 0.5, m).astype(np.float32)
    data, mask = _finish(vals, idx, n)
    return Workload("sk_ok_large", dims, data, mask,
                    CovSpec(EXPONENTIAL, (30.0, 15.0, 6.0), (30.0, 0.0, 0.0), 1.0, 0.05),
                    (30, 15, 6), 32)


INDICATOR_MARGINALS = [0.40, 0.25, 0.15, 0.12, 0.08]


def indicator(scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(3)
    dims = _scaled_dims((200, 200, 100), scale)
    n = dims[0] * dims[1] * dims[2]
    field = gaussian_field(dims, (20.0, 20.0, 6.0), rng)
    cuts = np.quantile(field, np.cumsum(INDICATOR_MARGINALS)[:-1])
    cats = np.searchsorted(cuts, field, side="right").astype(np.uint8)
    m = max(1, int(n * 0.015))
    idx = rng.choice(n, m, replace=False)
    data = np.zeros(n, dtype=np.uint8)
    mask = np.zeros(n, dtype=np.uint8)
    data[idx] = cats[idx]
    mask[idx] = 1
    covs, rads = [], []
    for c in range(5):
        a = 12.0 + 13.0 * c / 4.0
        covs.append(CovSpec(SPHERICAL, (a, a, 4.0 + c), (0.0, 0.0, 0.0), 1.0, 0.05 + 0.025 * c))
        rads.append((int(round(a)), int(round(a)), 4 + c))
    return Workload("indicator", dims, data, mask, covs[2], rads[2], 24, categories=5,
                    marginals=list(INDICATOR_MARGINALS), cat_covs=covs, cat_radiuses=rads)


def gauss_cv(scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(4)
    dims = _scaled_dims((200, 200, 50), scale)
    n = dims[0] * dims[1] * dims[2]
    field = gaussian_field(dims, (18.0, 18.0, 6.0), rng)
    m = max(1, int(round(4000 * n / 2000000)))
    idx = rng.choice(n, m, replace=False)
    data, mask = _finish(field[idx], idx, n)
    return Workload("gauss_cv", dims, data, mask,
                    CovSpec(GAUSSIAN, (18.0, 18.0, 6.0), (0.0, 0.0, 0.0), 1.0, 0.05),
                    (18, 18, 6), 24)


def clustered(scale: float = 1.0) -> Workload:
    rng = np.random.default_rng(5)
    dims = _scaled_dims((512, 512, 64), scale)
    nx, ny, nz = dims
    n = nx * ny * nz
    m = max(1, int(n * 0.002))
    centres = np.stack([rng.uniform(0, d, 50) for d in dims], axis=1)
    taken = set()
    idx = []
    while len(idx) < m:
        c = centres[rng.integers(0, 50)]
        p = np.rint(c + rng.normal(0.0, 8.0, 3)).astype(np.int64)
        if np.any(p < 0) or p[0] >= nx or p[1] >= ny or p[2] >= nz:
            continue
        node = int(p[0] + nx * p[1] + nx * ny * p[2])
        if node in taken:
            continue
        taken.add(node)
        idx.append(node)
    idx = np.array(idx, dtype=np.int64)
    vals = rng.standard_normal(m).astype(np.float32)
    data, mask = _finish(vals, idx, n)
    return Workload("clustered", dims, data, mask,
                    CovSpec(GAUSSIAN, (40.0, 40.0, 8.0), (0.0, 0.0, 0.0), 1.0, 1e-3),
                    (40, 40, 8), 64)


def lvm_means(dims, seed: int = 5) -> np.ndarray:
    """A smooth locally varying mean over the grid (flat, Fortran order): a
    plane plus a long-wavelength sine, the shape of the trend fields LVM
    kriging is run with."""
    nx, ny, nz = dims
    x, y, z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    rng = np.random.default_rng(seed)
    a, b, c = rng.uniform(-0.02, 0.02, 3)
    m = 0.3 + a * x + b * y + c * z + 0.4 * np.sin(2 * np.pi * x / max(nx, 2)) * np.cos(2 * np.pi * y / max(ny, 2))
    return m.reshape(-1, order="F").astype(np.float32)


ALL = {"ok_small": ok_small, "sk_ok_large": sk_ok_large, "indicator": indicator,
       "gauss_cv": gauss_cv, "clustered": clustered}
