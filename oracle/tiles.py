"""Tile-intersection oracle (numpy) -- TEST INFRASTRUCTURE ONLY.

Restates the reference's tile logic with IEEE arithmetic in the input
precision:
* tile bounds: ``IsectTilesKernel.cu:30-40`` (clamp) and ``:79-103``
  (floor((m - r)/T), ceil((m + r)/T), half-open), 3D ``IsectTiles3DKernel.cu:38-112``;
* records: key = camera * n_tiles + tile_y * tiles_x + tile_x, id = c*N + n,
  emitted per element in row-major tile order (``IsectTilesKernel.cu:137-217``);
  3D key = (tz * tiles_y + ty) * tiles_x + tx (``IsectTiles3DKernel.cu:147-227``);
* a stable sort by key (``IsectTilesKernel.cu:398-445``) -- ids ascend within a key;
* offsets[k] = number of keys < k (``IsectTilesKernel.cu:233-273``).

For power-of-two tile sizes the divisions are exact, so these integers equal
the CUDA path's bit for bit given the same projected centres and radii.
"""

from __future__ import annotations

import numpy as np


def _bound(value, upper):
    value = np.asarray(value)
    out = np.where(np.isfinite(value) & (value > 0), value, 0)
    out = np.minimum(out, upper)
    return out.astype(np.int64)


def tile_span(mean, radius, tile_size, n_tiles, dtype):
    t = dtype(tile_size)
    centre = np.asarray(mean, dtype=dtype) / t
    rad = np.asarray(radius, dtype=dtype) / t
    with np.errstate(invalid="ignore"):
        lo = _bound(np.floor(centre - rad), n_tiles)
        hi = _bound(np.ceil(centre + rad), n_tiles)
    return lo, hi


def isect_tiles_2d(means2d, radii, tile_size, tiles_x, tiles_y):
    """-> (tiles_per_gauss [C,N] int32, isect_ids int64, flatten_ids int32)."""
    means2d = np.asarray(means2d)
    radii = np.asarray(radii)
    dtype = means2d.dtype.type
    c, n = means2d.shape[:2]
    if radii.ndim == 2:
        radii = np.stack((radii, radii), axis=-1)
    mx, my = means2d[..., 0].reshape(-1), means2d[..., 1].reshape(-1)
    rx, ry = radii[..., 0].reshape(-1), radii[..., 1].reshape(-1)
    valid = (rx > 0) & (ry > 0) & np.isfinite(mx) & np.isfinite(my)
    x0, x1 = tile_span(mx, rx, tile_size, tiles_x, dtype)
    y0, y1 = tile_span(my, ry, tile_size, tiles_y, dtype)
    valid &= (x1 > x0) & (y1 > y0)
    counts = np.where(valid, (x1 - x0) * (y1 - y0), 0)
    keys, ids = [], []
    n_tiles = tiles_x * tiles_y
    for idx in np.nonzero(counts)[0]:
        cam = idx // n
        yy, xx = np.meshgrid(np.arange(y0[idx], y1[idx]), np.arange(x0[idx], x1[idx]), indexing="ij")
        keys.append(cam * n_tiles + (yy * tiles_x + xx).reshape(-1))
        ids.append(np.full(yy.size, idx, dtype=np.int64))
    keys = np.concatenate(keys) if keys else np.zeros(0, np.int64)
    ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
    order = np.argsort(keys, kind="stable")
    return counts.reshape(c, n).astype(np.int32), keys[order].astype(np.int64), ids[order].astype(np.int32)


def isect_tiles_3d(means3d, radii, tile_size, tiles_x, tiles_y, tiles_z):
    means3d = np.asarray(means3d)
    radii = np.asarray(radii)
    dtype = means3d.dtype.type
    valid = np.all(radii > 0, axis=1)
    spans = [tile_span(means3d[:, a], radii[:, a], tile_size, t, dtype)
             for a, t in enumerate((tiles_x, tiles_y, tiles_z))]
    for lo, hi in spans:
        valid &= hi > lo
    counts = np.where(valid, np.prod([hi - lo for lo, hi in spans], axis=0), 0)
    keys, ids = [], []
    for idx in np.nonzero(counts)[0]:
        (x0, x1), (y0, y1), (z0, z1) = ((lo[idx], hi[idx]) for lo, hi in spans)
        zz, yy, xx = np.meshgrid(np.arange(z0, z1), np.arange(y0, y1), np.arange(x0, x1), indexing="ij")
        keys.append(((zz * tiles_y + yy) * tiles_x + xx).reshape(-1))
        ids.append(np.full(zz.size, idx, dtype=np.int64))
    keys = np.concatenate(keys) if keys else np.zeros(0, np.int64)
    ids = np.concatenate(ids) if ids else np.zeros(0, np.int64)
    order = np.argsort(keys, kind="stable")
    return counts.astype(np.int32), keys[order].astype(np.int64), ids[order].astype(np.int32)


def offset_encode(isect_ids, n_keys):
    return np.searchsorted(np.asarray(isect_ids, dtype=np.int64), np.arange(n_keys), side="left").astype(np.int32)


__all__ = ["isect_tiles_2d", "isect_tiles_3d", "offset_encode", "tile_span"]
