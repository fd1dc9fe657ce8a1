"""Seeded synthetic rasters for the benchmark workloads (the reference publishes no dataset for this path).

All rasters are float64, row-major, NaN = NoData, drawn with ``numpy.random.default_rng(seed)``.

* ``omni_128``  -- 128 x 128, resistance exp(N(0, 1)) clipped to [1, 100], source 1 / resistance; radius 8,
  block 1, 8 neighbours, average-conductance edges; cumulative current, flow potential, normalised current.
* ``omni_1024`` -- 1024 x 1024 Gaussian random field g (power spectrum ~ |k|^-3, rescaled to [0, 1]),
  resistance 10^(2 g) in [1, 100], about 1% NoData as random 3 x 3 clusters, source 1 where g < 0.3;
  radius 32, block 3.
* ``adjoint_512`` -- 512 x 512, the resistance of ``omni_1024`` (field, 1% NoData clusters), Omniscape's
  default sources 1 / resistance (held fixed when differentiating); radius 24, block 1; J = sum of the
  cumulative current over rows and columns 224-287.
* ``omni_4096`` -- 4096 x 4096 field with exponent -2.5, resistance 500^g in [1, 500], 5% NoData as random
  polygons, source 1 / resistance above the 40th percentile of resistance, else 0; radius 64, block 5.
* ``advanced_rasters`` -- independent grounded raster circuits (the advanced mode): sides drawn uniformly from
  64 to 512, resistance log-uniform in [1, 1000] (conductance 1 / resistance), one unit current source and one
  direct ground at two distinct random cells; 4 neighbours.
"""

from __future__ import annotations

import numpy as np


def gaussian_field(n: int, exponent: float, seed: int, m: int | None = None) -> np.ndarray:
    """White noise filtered to a power spectrum ~ |k|^exponent, rescaled to [0, 1] (n rows x m columns)."""
    m = n if m is None else m
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n, m))
    ky = np.fft.fftfreq(n)[:, None]
    kx = np.fft.rfftfreq(m)[None, :]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = np.inf
    g = np.fft.irfft2(np.fft.rfft2(w) * k ** (exponent / 2.0), s=(n, m))
    return (g - g.min()) / (g.max() - g.min())


def nodata_clusters(shape, fraction: float, seed: int, size: int = 3) -> np.ndarray:
    """Mask of round(fraction * cells / size^2) random size x size clusters (seeded centres)."""
    rng = np.random.default_rng(seed)
    ny, nx = shape
    count = int(round(fraction * ny * nx / (size * size)))
    mask = np.zeros(shape, dtype=bool)
    h = size // 2
    ys = rng.integers(0, ny, count)
    xs = rng.integers(0, nx, count)
    for dy in range(-h, size - h):
        for dx in range(-h, size - h):
            mask[np.clip(ys + dy, 0, ny - 1), np.clip(xs + dx, 0, nx - 1)] = True
    return mask


def nodata_polygons(shape, fraction: float, seed: int) -> np.ndarray:
    """Random convex polygons (5-9 vertices, radii 3-40 cells) until about `fraction` of the cells are covered."""
    rng = np.random.default_rng(seed)
    ny, nx = shape
    mask = np.zeros(shape, dtype=bool)
    target = fraction * ny * nx
    covered = 0
    while covered < target:
        cy, cx = rng.uniform(0, ny), rng.uniform(0, nx)
        rad = rng.uniform(3, 40)
        k = int(rng.integers(5, 10))
        ang = np.sort(rng.uniform(0, 2 * np.pi, k))
        rr = rad * rng.uniform(0.6, 1.0, k)
        py, px = cy + rr * np.sin(ang), cx + rr * np.cos(ang)
        y0, y1 = int(max(0, np.floor(py.min()))), int(min(ny - 1, np.ceil(py.max())))
        x0, x1 = int(max(0, np.floor(px.min()))), int(min(nx - 1, np.ceil(px.max())))
        if y1 < y0 or x1 < x0:
            continue
        yy, xx = np.mgrid[y0:y1 + 1, x0:x1 + 1]
        inside = np.ones(yy.shape, dtype=bool)
        for i in range(k):  # convex polygon, vertices counter-clockwise in (x, y)
            ax, ay, bx, by = px[i], py[i], px[(i + 1) % k], py[(i + 1) % k]
            inside &= (bx - ax) * (yy - ay) - (by - ay) * (xx - ax) >= 0
        before = mask[y0:y1 + 1, x0:x1 + 1].sum()
        mask[y0:y1 + 1, x0:x1 + 1] |= inside
        covered += mask[y0:y1 + 1, x0:x1 + 1].sum() - before
    return mask


def omni_128(seed: int = 0):
    rng = np.random.default_rng(seed)
    r = np.clip(np.exp(rng.normal(0.0, 1.0, (128, 128))), 1.0, 100.0)
    return r, 1.0 / r, dict(radius=8, block_size=1, buffer=0, four_neighbors=False, flow_potential=True,
                           normalized_current=True)


def omni_grf(n: int, seed: int = 0, nodata: float = 0.01):
    g = gaussian_field(n, -3.0, seed)
    r = 10.0 ** (2.0 * g)
    r[nodata_clusters(r.shape, nodata, seed + 1)] = np.nan
    s = np.where(g < 0.3, 1.0, 0.0)
    return r, s


def omni_1024(seed: int = 0):
    r, s = omni_grf(1024, seed)
    return r, s, dict(radius=32, block_size=3, buffer=0, four_neighbors=False)


def adjoint_512(seed: int = 0):
    r, _ = omni_grf(512, seed)
    s = np.where(np.isnan(r), 0.0, 1.0 / np.nan_to_num(r, nan=1.0))  # Omniscape's default sources, 1 / resistance
    weight = np.zeros(r.shape)
    weight[224:288, 224:288] = 1.0
    return r, s, weight, dict(radius=24, block_size=1, buffer=0, four_neighbors=False)


def omni_4096(seed: int = 0):
    g = gaussian_field(4096, -2.5, seed)
    r = 500.0 ** g
    r[nodata_polygons(r.shape, 0.05, seed + 1)] = np.nan
    p40 = np.nanpercentile(r, 40)
    s = np.where(r > p40, 1.0 / r, 0.0)
    s[np.isnan(s)] = 0.0
    return r, s, dict(radius=64, block_size=5, buffer=0, four_neighbors=False)


def pairwise_256(seed: int = 0, n_points: int = 24):
    """Circuitscape pairwise workload: a 256 x 256 resistance raster (the Omniscape workloads' Gaussian random field,
    r = 10^(2g) in [1, 100], 1% NoData in 3 x 3 clusters) and `n_points` focal points with ids 1..n_points on
    distinct random cells with data.  Returns (resistance with NaN NoData, point raster)."""
    r, _ = omni_grf(256, seed)
    rng = np.random.default_rng(seed + 7)
    ok = np.flatnonzero(np.isfinite(r).ravel())
    pm = np.zeros(r.shape)
    pm.flat[rng.choice(ok, size=n_points, replace=False)] = np.arange(1, n_points + 1)
    return r, pm


def _advanced_draws(rng, side_min, side_max):
    ny, nx = (int(v) for v in rng.integers(side_min, side_max + 1, 2))
    r = np.exp(rng.uniform(np.log(1.0), np.log(1000.0), (ny, nx)))
    a, b = rng.choice(ny * nx, 2, replace=False)
    return ny, nx, r, int(a), int(b)


def advanced_rasters(n=4096, seed=0, side_min=64, side_max=512):
    """(conductance, source, ground) triples of the advanced-mode batch."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        ny, nx, r, a, b = _advanced_draws(rng, side_min, side_max)
        s = np.zeros((ny, nx))
        gr = np.zeros((ny, nx))
        s.flat[a] = 1.0
        gr.flat[b] = np.inf
        out.append((1.0 / r, s, gr))
    return out


def advanced_packed(n=4096, seed=0, side_min=64, side_max=512):
    """The same rasters as advanced_rasters, packed back to back: (shapes, conductance, source, ground)."""
    rng = np.random.default_rng(seed)
    shapes, gs, src, gnd = [], [], [], []
    off = 0
    for _ in range(n):
        ny, nx, r, a, b = _advanced_draws(rng, side_min, side_max)
        shapes.append((ny, nx))
        gs.append((1.0 / r).ravel())
        src.append(off + a)
        gnd.append(off + b)
        off += ny * nx
    g = np.concatenate(gs)
    del gs
    s = np.zeros(off)
    gr = np.zeros(off)
    s[src] = 1.0
    gr[gnd] = np.inf
    return shapes, g, s, gr


WORKLOADS = {"omni_128": omni_128, "omni_1024": omni_1024, "omni_4096": omni_4096}
