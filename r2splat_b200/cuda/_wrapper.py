"""Low-level operator surface of r2splat_b200.

Same names, argument order and return tuples as the reference's low-level
surface (``r2splat/cuda/_wrapper.py:19-165``, bound from ``ext.cpp:8-183``, with
signatures in ``Ops.h:13-456``). Each function validates like the reference's
C++ wrappers (RuntimeError for shape / dtype / device errors), allocates its
outputs with the torch caching allocator, and enqueues one C-ABI call on the
current stream of the inputs' device.
"""

from __future__ import annotations

import ctypes
import math
from typing import Optional

import torch

from . import _backend

Tensor = torch.Tensor
_VOID = ctypes.c_void_p


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def _ptr(t: Optional[Tensor]):
    return None if t is None else _VOID(t.data_ptr())


def _stream(device: torch.device):
    return _VOID(torch.cuda.current_stream(device).cuda_stream)


def _dtype(t: Tensor) -> int:
    if t.dtype == torch.float32:
        return 0
    if t.dtype == torch.float64:
        return 1
    raise RuntimeError(f"expected float32 or float64 tensors, got {t.dtype}")


def _check(name: str, t: Tensor, device: Optional[torch.device] = None) -> None:
    if not isinstance(t, Tensor):
        raise RuntimeError(f"{name} must be a tensor")
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if not t.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")
    if device is not None and t.device != device:
        raise RuntimeError(f"{name} must be on the same CUDA device as the other inputs")


def _check_float(name: str, t: Tensor, like: Tensor) -> None:
    _check(name, t, like.device)
    if t.dtype != like.dtype:
        raise RuntimeError(f"{name} must have the same dtype as the other inputs")


def _require(cond: bool, message: str) -> None:
    if not cond:
        raise RuntimeError(message)


def _workspace(nbytes: int, device: torch.device) -> Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


class _Guard:
    """Runs on the inputs' device and restores the caller's current device."""

    def __init__(self, device: torch.device):
        self._ctx = torch.cuda.device(device)

    def __enter__(self):
        self._ctx.__enter__()
        return self

    def __exit__(self, *exc):
        return self._ctx.__exit__(*exc)


# ---------------------------------------------------------------------------
# parameter transform / projection / conics
# ---------------------------------------------------------------------------

def parameter_transform_fwd(quats: Tensor, scales: Tensor):
    """Normalise wxyz quaternions and form covariance from physical scales.

    quats [N,4], scales [N,3] -> (covars [N,6] packed (00,01,02,11,12,22), max_scales [N]).
    """
    _check("quats", quats)
    _check("scales", scales)
    _require(quats.dim() == 2 and quats.size(1) == 4, f"quats must have shape [N, 4], got {list(quats.shape)}")
    _require(scales.dim() == 2 and scales.size(1) == 3, f"scales must have shape [N, 3], got {list(scales.shape)}")
    _dtype(quats)
    _require(scales.dtype == quats.dtype, "scales must have the same dtype as quats")
    _require(scales.device == quats.device, "scales must be on the same CUDA device as quats")
    _require(scales.size(0) == quats.size(0), "scales and quats must have the same batch size")
    n = quats.size(0)
    covars = quats.new_empty((n, 6))
    max_scales = quats.new_empty((n,))
    if n:
        with _Guard(quats.device):
            _backend.call("r2s_parameter_transform_fwd", _dtype(quats), _ptr(quats), _ptr(scales), _ptr(covars),
                          _ptr(max_scales), n, _stream(quats.device))
    return covars, max_scales


def parameter_transform_bwd(quats: Tensor, scales: Tensor, v_covars: Tensor):
    """VJP to raw quaternions and physical scales from packed covariance adjoints [N,6]."""
    _check("quats", quats)
    _check("scales", scales)
    _require(quats.dim() == 2 and quats.size(1) == 4, f"quats must have shape [N, 4], got {list(quats.shape)}")
    _require(scales.dim() == 2 and scales.size(1) == 3, f"scales must have shape [N, 3], got {list(scales.shape)}")
    _dtype(quats)
    _require(scales.dtype == quats.dtype, "scales must have the same dtype as quats")
    _require(scales.device == quats.device, "scales must be on the same CUDA device as quats")
    _require(scales.size(0) == quats.size(0), "scales and quats must have the same batch size")
    _check("v_covars", v_covars)
    _require(v_covars.dim() == 2 and v_covars.size(1) == 6 and v_covars.size(0) == quats.size(0),
             f"v_covars must have shape [N, 6], got {list(v_covars.shape)}")
    _require(v_covars.dtype == quats.dtype, "v_covars must have the same dtype as quats")
    _require(v_covars.device == quats.device, "v_covars must be on the same CUDA device as quats")
    n = quats.size(0)
    v_quats = quats.new_empty((n, 4))
    v_scales = quats.new_empty((n, 3))
    if n:
        with _Guard(quats.device):
            _backend.call("r2s_parameter_transform_bwd", _dtype(quats), _ptr(quats), _ptr(scales), _ptr(v_covars),
                          _ptr(v_quats), _ptr(v_scales), n, _stream(quats.device))
    return v_quats, v_scales


def world_to_image_projection_fwd(means, covars, viewmats, Ks, dim1, dim0, eps_blur, radius_clip):
    """Project [N] world primitives into [C] pinhole cameras.

    -> (means2d [C,N,2], cov2d [C,N,6] (pixel x, pixel y, ray axis), radii [C,N,2] int32).
    ``eps_blur`` and ``radius_clip`` are single-precision arguments, as in the reference.
    """
    for name, t in (("means", means), ("covars", covars), ("viewmats", viewmats), ("Ks", Ks)):
        _check(name, t, means.device)
    _require(means.dim() == 2 and means.size(1) == 3, f"means must be 2D [N, 3], got shape {list(means.shape)}")
    _require(covars.dim() == 2 and covars.size(1) == 6, f"covars must be 2D [N, 6], got shape {list(covars.shape)}")
    _require(viewmats.dim() == 3 and viewmats.shape[1:] == (4, 4),
             f"viewmats must be 3D [C, 4, 4], got shape {list(viewmats.shape)}")
    _require(Ks.dim() == 3 and Ks.shape[1:] == (3, 3), f"Ks must be 3D [C, 3, 3], got shape {list(Ks.shape)}")
    _require(float(radius_clip) > 0, f"radius_clip must be positive, got {radius_clip}")
    n, c = means.size(0), viewmats.size(0)
    _require(covars.size(0) == n, f"covars dim 0 ({covars.size(0)}) doesn't match N={n}")
    _require(Ks.size(0) == c, f"Ks batch dim ({Ks.size(0)}) doesn't match C={c}")
    for t in (covars, viewmats, Ks):
        _require(t.dtype == means.dtype, "inputs must share one dtype")
    means2d = means.new_empty((c, n, 2))
    cov2d = means.new_empty((c, n, 6))
    radii = torch.zeros((c, n, 2), dtype=torch.int32, device=means.device)
    if c * n:
        with _Guard(means.device):
            _backend.call("r2s_world_to_image_projection_fwd", _dtype(means), _ptr(means), _ptr(covars),
                          _ptr(viewmats), _ptr(Ks), c, n, int(dim1), int(dim0), float(eps_blur), float(radius_clip),
                          _ptr(means2d), _ptr(cov2d), _ptr(radii), _stream(means.device))
    return means2d, cov2d, radii


def world_to_image_projection_bwd(means, covars, viewmats, Ks, dim1, dim0, v_means2d, v_cov2d_3x3):
    """VJP of the projection to (v_means [N,3], v_covars [N,6]), summed over cameras."""
    for name, t in (("means", means), ("covars", covars), ("viewmats", viewmats), ("Ks", Ks),
                    ("v_means2d", v_means2d), ("v_cov2d_3x3", v_cov2d_3x3)):
        _check(name, t, means.device)
    n, c = means.size(0), viewmats.size(0)
    _require(means.dim() == 2 and means.size(1) == 3, "means must be 2D [N, 3]")
    _require(covars.shape == (n, 6), "covars must be 2D [N, 6]")
    _require(v_means2d.shape == (c, n, 2), "v_means2d must be [C, N, 2]")
    _require(v_cov2d_3x3.shape == (c, n, 6), "v_cov2d_3x3 must be [C, N, 6]")
    v_means = means.new_empty((n, 3))
    v_covars = means.new_empty((n, 6))
    if n:
        with _Guard(means.device):
            _backend.call("r2s_world_to_image_projection_bwd", _dtype(means), _ptr(means), _ptr(covars),
                          _ptr(viewmats), _ptr(Ks), c, n, int(dim1), int(dim0), _ptr(v_means2d), _ptr(v_cov2d_3x3),
                          _ptr(v_means), _ptr(v_covars), _stream(means.device))
    return v_means, v_covars


def conics_mu_fwd(cov2d_3x3: Tensor, eps: float):
    """Conic of the blurred 2x2 footprint and the Gaussian path factor mu.

    cov2d [C,N,6] -> (conics [C,N,3], mus [C,N]).
    """
    _check("cov2d_3x3", cov2d_3x3)
    _require(cov2d_3x3.dim() == 3 and cov2d_3x3.size(2) == 6, "cov2d_3x3 must be 3D [C, N, 6]")
    c, n = cov2d_3x3.shape[:2]
    conics = cov2d_3x3.new_empty((c, n, 3))
    mus = cov2d_3x3.new_empty((c, n))
    if c * n:
        with _Guard(cov2d_3x3.device):
            _backend.call("r2s_conics_mu_fwd", _dtype(cov2d_3x3), _ptr(cov2d_3x3), c * n, float(eps), _ptr(conics),
                          _ptr(mus), _stream(cov2d_3x3.device))
    return conics, mus


def conics_mu_bwd(cov2d_3x3, eps, conics, mus, v_conics, v_mus):
    """VJP of conics_mu_fwd from the saved conics and mus -> v_cov2d [C,N,6]."""
    for name, t in (("cov2d_3x3", cov2d_3x3), ("conics", conics), ("mus", mus), ("v_conics", v_conics),
                    ("v_mus", v_mus)):
        _check(name, t, cov2d_3x3.device)
    _require(cov2d_3x3.dim() == 3 and cov2d_3x3.size(2) == 6, "cov2d_3x3 must be 3D [C, N, 6]")
    c, n = cov2d_3x3.shape[:2]
    _require(conics.shape == (c, n, 3), "conics shape must be [C, N, 3]")
    _require(mus.shape == (c, n), "mus shape must be [C, N]")
    _require(v_conics.shape == (c, n, 3), "v_conics shape must be [C, N, 3]")
    _require(v_mus.shape == (c, n), "v_mus shape must be [C, N]")
    out = cov2d_3x3.new_empty((c, n, 6))
    if c * n:
        with _Guard(cov2d_3x3.device):
            _backend.call("r2s_conics_mu_bwd", _dtype(cov2d_3x3), _ptr(cov2d_3x3), c * n, float(eps), _ptr(conics),
                          _ptr(mus), _ptr(v_conics), _ptr(v_mus), _ptr(out), _stream(cov2d_3x3.device))
    return out


def world_to_volume_mapping_fwd(means, covars, max_scales, ranges, centers, dim2, dim1, dim0, eps3d, radius_clip):
    """Affine world -> voxel mapping: (means3d_v [N,3], conics [N,6], radii [N,3] int32)."""
    for name, t in (("means", means), ("covars", covars), ("max_scales", max_scales), ("ranges", ranges),
                    ("centers", centers)):
        _check(name, t, means.device)
    _require(means.dim() == 2 and means.size(1) == 3, f"means must be 2D [N, 3], got shape {list(means.shape)}")
    _require(covars.dim() == 2 and covars.size(1) == 6, f"covars must be 2D [N, 6], got shape {list(covars.shape)}")
    _require(max_scales.dim() == 1, f"max_scales must be 1D [N], got dim {max_scales.dim()}")
    _require(ranges.shape == (3,), f"ranges must be 1D [3], got shape {list(ranges.shape)}")
    _require(centers.shape == (3,), f"centers must be 1D [3], got shape {list(centers.shape)}")
    n = means.size(0)
    _require(covars.size(0) == n, f"covars batch dim ({covars.size(0)}) doesn't match N={n}")
    _require(max_scales.size(0) == n, f"max_scales batch dim ({max_scales.size(0)}) doesn't match N={n}")
    means_v = means.new_empty((n, 3))
    conics = means.new_empty((n, 6))
    radii = torch.empty((n, 3), dtype=torch.int32, device=means.device)
    if n:
        with _Guard(means.device):
            _backend.call("r2s_world_to_volume_mapping_fwd", _dtype(means), _ptr(means), _ptr(covars), _ptr(ranges),
                          _ptr(centers), n, int(dim2), int(dim1), int(dim0), float(eps3d), float(radius_clip),
                          _ptr(means_v), _ptr(conics), _ptr(radii), _stream(means.device))
    return means_v, conics, radii


def world_to_volume_mapping_bwd(means, covars, ranges, centers, dim2, dim1, dim0, eps3d, v_means3d_v, v_conics):
    """VJP of the volume mapping: (v_means [N,3], v_covars [N,6])."""
    for name, t in (("means", means), ("covars", covars), ("ranges", ranges), ("centers", centers),
                    ("v_means3d_v", v_means3d_v), ("v_conics", v_conics)):
        _check(name, t, means.device)
    n = means.size(0)
    _require(v_means3d_v.shape == (n, 3), "v_means3d_v must be [N, 3]")
    _require(v_conics.shape == (n, 6), "v_conics must be [N, 6]")
    v_means = means.new_empty((n, 3))
    v_covars = means.new_empty((n, 6))
    if n:
        with _Guard(means.device):
            _backend.call("r2s_world_to_volume_mapping_bwd", _dtype(means), _ptr(means), _ptr(covars), _ptr(ranges),
                          _ptr(centers), n, int(dim2), int(dim1), int(dim0), float(eps3d), _ptr(v_means3d_v),
                          _ptr(v_conics), _ptr(v_means), _ptr(v_covars), _stream(means.device))
    return v_means, v_covars


# ---------------------------------------------------------------------------
# tile intersection
# ---------------------------------------------------------------------------

def _total(cum: Tensor) -> int:
    # One device->host read of the intersection count (the reference reads it
    # with .item() as well, IsectTiles.cpp:99-100).
    return int(cum[-1].item()) if cum.numel() else 0


def isect_tiles(means2d: Tensor, radii: Tensor, tile_size: int, n_tiles_dim1: int, n_tiles_dim0: int):
    """2D tile intersections sorted by (camera, tile) with ids ascending within a tile.

    means2d [C,N,2], radii [C,N] or [C,N,2] int32 ->
    (tiles_per_gauss [C,N] int32, isect_ids [M] int64, flatten_ids [M] int32).
    """
    _check("means2d", means2d)
    _check("radii", radii, means2d.device)
    _require(means2d.dim() == 3, "means2d must be 3D [C, N, 2]")
    _require(radii.dim() == 2 or (radii.dim() == 3 and radii.size(2) == 2), "radii must be 2D [C, N] or 3D [C, N, 2]")
    _require(means2d.size(2) == 2, "means2d last dim must be 2")
    _require(means2d.size(0) == radii.size(0), "C dimension must match")
    _require(means2d.size(1) == radii.size(1), "N dimension must match")
    _require(radii.dtype == torch.int32, "radii must be int32")
    c, n = means2d.shape[:2]
    device = means2d.device
    tiles_per_gauss = torch.empty((c, n), dtype=torch.int32, device=device)
    empty64 = torch.empty((0,), dtype=torch.int64, device=device)
    empty32 = torch.empty((0,), dtype=torch.int32, device=device)
    if c * n == 0:
        return tiles_per_gauss, empty64, empty32
    rect = 1 if radii.dim() == 3 else 0
    tx, ty = int(n_tiles_dim1), int(n_tiles_dim0)
    with _Guard(device):
        stream = _stream(device)
        cum = torch.empty((c * n,), dtype=torch.int64, device=device)
        lib = _backend.library()
        ws = _workspace(lib.r2s_isect_count_workspace(c * n), device)
        _backend.call("r2s_isect_tiles_count", _dtype(means2d), _ptr(means2d), _ptr(radii), rect, c, n,
                      int(tile_size), tx, ty, _ptr(tiles_per_gauss), _ptr(cum), _ptr(ws), ws.numel(), stream)
        m = _total(cum)
        if m == 0:
            return tiles_per_gauss, empty64, empty32
        isect_ids = torch.empty((m,), dtype=torch.int64, device=device)
        flatten_ids = torch.empty((m,), dtype=torch.int32, device=device)
        ws = _workspace(lib.r2s_isect_emit_workspace(m, c * tx * ty), device)
        _backend.call("r2s_isect_tiles_emit", _dtype(means2d), _ptr(means2d), _ptr(radii), rect, c, n,
                      int(tile_size), tx, ty, _ptr(cum), m, _ptr(isect_ids), _ptr(flatten_ids), None, _ptr(ws),
                      ws.numel(), stream)
    return tiles_per_gauss, isect_ids, flatten_ids


def isect_offset_encode(isect_ids: Tensor, C: int, n_tiles_dim1: int, n_tiles_dim0: int):
    """Per-(camera, tile) start offsets of sorted isect_ids -> [C, tiles_y, tiles_x] int32."""
    _check("isect_ids", isect_ids)
    offsets = torch.empty((int(C), int(n_tiles_dim0), int(n_tiles_dim1)), dtype=torch.int32, device=isect_ids.device)
    if offsets.numel():
        with _Guard(isect_ids.device):
            _backend.call("r2s_isect_offset_encode", _ptr(isect_ids), isect_ids.numel(), int(C), int(n_tiles_dim1),
                          int(n_tiles_dim0), _ptr(offsets), _stream(isect_ids.device))
    return offsets


def isect_tiles_3d(means3d: Tensor, radii: Tensor, tile_size: int, n_tiles_dim2: int, n_tiles_dim1: int,
                   n_tiles_dim0: int):
    """3D tile intersections sorted by tile id (x fastest) with ids ascending within a tile."""
    _check("means3d", means3d)
    _check("radii", radii, means3d.device)
    _require(means3d.dim() == 2 and means3d.size(1) == 3, "means3d must be 2D [N, 3]")
    _require(radii.dim() == 2 and radii.size(1) == 3, "radii must be 2D [N, 3]")
    _require(radii.size(0) == means3d.size(0), "N dimension must match")
    _require(radii.dtype == torch.int32, "radii must be int32")
    n = means3d.size(0)
    device = means3d.device
    tiles_per_gauss = torch.empty((n,), dtype=torch.int32, device=device)
    empty64 = torch.empty((0,), dtype=torch.int64, device=device)
    empty32 = torch.empty((0,), dtype=torch.int32, device=device)
    if n == 0:
        return tiles_per_gauss, empty64, empty32
    tx, ty, tz = int(n_tiles_dim2), int(n_tiles_dim1), int(n_tiles_dim0)
    with _Guard(device):
        stream = _stream(device)
        cum = torch.empty((n,), dtype=torch.int64, device=device)
        lib = _backend.library()
        ws = _workspace(lib.r2s_isect_count_workspace(n), device)
        _backend.call("r2s_isect_tiles_3d_count", _dtype(means3d), _ptr(means3d), _ptr(radii), n, int(tile_size),
                      tx, ty, tz, _ptr(tiles_per_gauss), _ptr(cum), _ptr(ws), ws.numel(), stream)
        m = _total(cum)
        if m == 0:
            return tiles_per_gauss, empty64, empty32
        isect_ids = torch.empty((m,), dtype=torch.int64, device=device)
        flatten_ids = torch.empty((m,), dtype=torch.int32, device=device)
        ws = _workspace(lib.r2s_isect_emit_workspace(m, tx * ty * tz), device)
        _backend.call("r2s_isect_tiles_3d_emit", _dtype(means3d), _ptr(means3d), _ptr(radii), n, int(tile_size),
                      tx, ty, tz, _ptr(cum), m, _ptr(isect_ids), _ptr(flatten_ids), None, _ptr(ws), ws.numel(),
                      stream)
    return tiles_per_gauss, isect_ids, flatten_ids


def isect_offset_encode_3d(isect_ids: Tensor, n_tiles_dim2: int, n_tiles_dim1: int, n_tiles_dim0: int):
    """Per-tile start offsets of sorted 3D isect_ids -> [tiles_z, tiles_y, tiles_x] int32."""
    _check("isect_ids", isect_ids)
    offsets = torch.empty((int(n_tiles_dim0), int(n_tiles_dim1), int(n_tiles_dim2)), dtype=torch.int32,
                          device=isect_ids.device)
    if offsets.numel():
        with _Guard(isect_ids.device):
            _backend.call("r2s_isect_offset_encode_3d", _ptr(isect_ids), isect_ids.numel(), int(n_tiles_dim2),
                          int(n_tiles_dim1), int(n_tiles_dim0), _ptr(offsets), _stream(isect_ids.device))
    return offsets


# ---------------------------------------------------------------------------
# rasterization
# ---------------------------------------------------------------------------

def _raster_inputs(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids, isect_ids=None):
    _check("means2d", means2d)
    _dtype(means2d)
    for name, t in (("conics", conics), ("opacities", opacities), ("mus", mus)):
        _check_float(name, t, means2d)
    _check("tile_offsets", tile_offsets, means2d.device)
    _check("flatten_ids", flatten_ids, means2d.device)
    _require(means2d.dim() == 3, "means2d must be 3D [C, N, 2]")
    _require(conics.dim() == 3, "conics must be 3D [C, N, 3]")
    _require(opacities.dim() == 2, "opacities must be 2D [C, N]")
    _require(mus.dim() == 2, "mus must be 2D [C, N]")
    _require(tile_offsets.dim() == 3, "tile_offsets must be 3D [C, n_tiles_dim0, n_tiles_dim1]")
    _require(flatten_ids.dim() == 1, "flatten_ids must be 1D [n_isects]")
    _require(means2d.size(2) == 2, "means2d last dim must be 2")
    _require(conics.size(2) == 3, "conics last dim must be 3")
    c, n = means2d.shape[:2]
    _require(conics.shape[:2] == (c, n), "conics shape must match means2d [C, N, 3]")
    _require(opacities.shape == (c, n), "opacities shape must match [C, N]")
    _require(mus.shape == (c, n), "mus shape must match [C, N]")
    _require(tile_offsets.size(0) == c, "tile_offsets C dimension must match")
    if betas is not None:
        _check_float("betas", betas, means2d)
        _require(betas.dim() == 2, "betas must be 2D [C, N]")
        _require(betas.shape == (c, n), "betas shape must match [C, N]")
    if isect_ids is not None:
        _check("isect_ids", isect_ids, means2d.device)
        _require(isect_ids.dim() == 1, "isect_ids must be 1D [n_isects]")
        _require(isect_ids.dtype == torch.int64, "isect_ids must be int64")
        _require(isect_ids.size(0) == flatten_ids.size(0), "isect_ids and flatten_ids must have the same length")
    _require(tile_offsets.dtype == torch.int32 and flatten_ids.dtype == torch.int32,
             "tile_offsets and flatten_ids must be int32")
    return c, n, flatten_ids.size(0), tile_offsets.size(1), tile_offsets.size(2)


def _raster_forward(means2d, conics, opacities, mus, betas, uncertainties, tile_offsets, flatten_ids, dim1, dim0,
                    tile_size):
    c, n, m, ty, tx = _raster_inputs(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids)
    if uncertainties is not None:
        _check_float("uncertainties", uncertainties, means2d)
        _require(uncertainties.dim() == 1, "uncertainties must be 1D [N]")
        _require(uncertainties.size(0) == n, "uncertainties shape must be [N]")
    device = means2d.device
    render = means2d.new_empty((c, int(dim0), int(dim1)))
    render_var = torch.empty_like(render) if uncertainties is not None else None
    with _Guard(device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_raster_workspace(_dtype(means2d), c, n, 0), device)
        if uncertainties is None:
            _backend.call("r2s_rasterize_to_pixels_fwd", _dtype(means2d), _ptr(means2d), _ptr(conics),
                          _ptr(opacities), _ptr(mus), _ptr(betas), _ptr(tile_offsets), _ptr(flatten_ids), c, n, m,
                          int(dim1), int(dim0), int(tile_size), tx, ty, _ptr(render), _ptr(ws), ws.numel(),
                          _stream(device))
            return render
        _backend.call("r2s_rasterize_to_pixels_mean_var_fwd", _dtype(means2d), _ptr(means2d), _ptr(conics),
                      _ptr(opacities), _ptr(mus), _ptr(betas), _ptr(uncertainties), _ptr(tile_offsets),
                      _ptr(flatten_ids), c, n, m, int(dim1), int(dim0), int(tile_size), tx, ty, _ptr(render),
                      _ptr(render_var), _ptr(ws), ws.numel(), _stream(device))
    return render, render_var


def _raster_backward(means2d, conics, opacities, mus, betas, tile_offsets, isect_ids, flatten_ids, v_render,
                     v_render_var, uncertainties, dim1, dim0, tile_size, absgrad, with_unc):
    c, n, m, ty, tx = _raster_inputs(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids, isect_ids)
    device = means2d.device
    shape = (c, int(dim0), int(dim1))
    if v_render is not None:
        _check_float("v_render_output", v_render, means2d)
        _require(v_render.dim() == 3, "v_render_output must be 3D [C, dim0, dim1]")
        _require(tuple(v_render.shape) == shape, "v_render_output shape must be [C, dim0, dim1]")
    if v_render_var is not None:
        _check_float("v_render_var", v_render_var, means2d)
        _require(v_render_var.dim() == 3, "v_render_var must be 3D [C, dim0, dim1]")
        _require(tuple(v_render_var.shape) == shape, "v_render_var shape must be [C, dim0, dim1]")
    if uncertainties is not None:
        _check_float("uncertainties", uncertainties, means2d)
        _require(uncertainties.dim() == 1, "uncertainties must be 1D [N]")
        _require(uncertainties.size(0) == n, "uncertainties shape must match [N]")
    v_means2d = torch.empty_like(means2d)
    v_conics = torch.empty_like(conics)
    v_opacities = torch.empty_like(opacities)
    v_mus = torch.empty_like(mus)
    v_betas = torch.empty_like(betas) if betas is not None else None
    v_abs = torch.empty_like(means2d) if absgrad else None
    v_unc = means2d.new_empty((n,)) if with_unc else None
    with _Guard(device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_raster_workspace(_dtype(means2d), c, n, 1), device)
        _backend.call("r2s_rasterize_to_pixels_bwd", _dtype(means2d), _ptr(means2d), _ptr(conics), _ptr(opacities),
                      _ptr(mus), _ptr(betas), _ptr(tile_offsets), _ptr(isect_ids), _ptr(flatten_ids),
                      _ptr(v_render), _ptr(v_render_var), _ptr(uncertainties), c, n, m, int(dim1), int(dim0),
                      int(tile_size), tx, ty, _ptr(v_abs), _ptr(v_means2d), _ptr(v_conics), _ptr(v_opacities),
                      _ptr(v_mus), _ptr(v_betas), _ptr(v_unc), _ptr(ws), ws.numel(), _stream(device))
    out = (v_abs, v_means2d, v_conics, v_opacities, v_mus)
    if betas is not None:
        out += (v_betas,)
    if with_unc:
        out += (v_unc,)
    return out


def rasterize_to_pixels_fwd(means2d, conics, opacities, mus, tile_offsets, flatten_ids, dim1, dim0, tile_size):
    """Additive Gaussian line integrals per pixel -> render [C, dim0, dim1]."""
    return _raster_forward(means2d, conics, opacities, mus, None, None, tile_offsets, flatten_ids, dim1, dim0,
                           tile_size)


def rasterize_to_pixels_mean_var_fwd(means2d, conics, opacities, mus, uncertainties, tile_offsets, flatten_ids,
                                     dim1, dim0, tile_size):
    """Gaussian mean image and propagated variance image (sum of q * alpha^2)."""
    return _raster_forward(means2d, conics, opacities, mus, None, uncertainties, tile_offsets, flatten_ids, dim1,
                           dim0, tile_size)


def beta_rasterize_to_pixels_fwd(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids, dim1, dim0,
                                 tile_size):
    """Additive Beta line integrals per pixel (betas = projected exponent beta + 1/2)."""
    return _raster_forward(means2d, conics, opacities, mus, betas, None, tile_offsets, flatten_ids, dim1, dim0,
                           tile_size)


def beta_rasterize_to_pixels_mean_var_fwd(means2d, conics, opacities, mus, betas, uncertainties, tile_offsets,
                                          flatten_ids, dim1, dim0, tile_size):
    return _raster_forward(means2d, conics, opacities, mus, betas, uncertainties, tile_offsets, flatten_ids, dim1,
                           dim0, tile_size)


def _uncertainty_bwd(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids, v_render_var, dim1, dim0,
                     tile_size):
    c, n, m, ty, tx = _raster_inputs(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids)
    _check_float("v_render_var", v_render_var, means2d)
    _require(v_render_var.dim() == 3, "v_render_var must be 3D [C, dim0, dim1]")
    _require(tuple(v_render_var.shape) == (c, int(dim0), int(dim1)), "v_render_var shape must be [C, dim0, dim1]")
    device = means2d.device
    v_unc = means2d.new_empty((n,))
    with _Guard(device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_raster_workspace(_dtype(means2d), c, n, 0), device)
        _backend.call("r2s_rasterize_to_pixels_uncertainty_bwd", _dtype(means2d), _ptr(means2d), _ptr(conics),
                      _ptr(opacities), _ptr(mus), _ptr(betas), _ptr(tile_offsets), _ptr(flatten_ids),
                      _ptr(v_render_var), c, n, m, int(dim1), int(dim0), int(tile_size), tx, ty, _ptr(v_unc),
                      _ptr(ws), ws.numel(), _stream(device))
    return v_unc


def rasterize_to_pixels_uncertainty_bwd(means2d, conics, opacities, mus, tile_offsets, flatten_ids, v_render_var,
                                        dim1, dim0, tile_size):
    """VJP of the variance image with respect to the per-primitive uncertainty [N]."""
    return _uncertainty_bwd(means2d, conics, opacities, mus, None, tile_offsets, flatten_ids, v_render_var, dim1,
                            dim0, tile_size)


def beta_rasterize_to_pixels_uncertainty_bwd(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids,
                                             v_render_var, dim1, dim0, tile_size):
    return _uncertainty_bwd(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids, v_render_var, dim1,
                            dim0, tile_size)


def rasterize_to_pixels_bwd(means2d, conics, opacities, mus, tile_offsets, flatten_ids, v_render_output, dim1, dim0,
                            tile_size, absgrad):
    """VJP of the image ("pixel" mode entry): (absgrad|None, v_means2d, v_conics, v_opacities, v_mus)."""
    return _raster_backward(means2d, conics, opacities, mus, None, tile_offsets, None, flatten_ids, v_render_output,
                            None, None, dim1, dim0, tile_size, absgrad, False)


def rasterize_to_pixels_bwd_per_gaussian(means2d, conics, opacities, mus, tile_offsets, isect_ids, flatten_ids,
                                         v_render_output, dim1, dim0, tile_size, absgrad):
    """VJP of the image ("primitive" mode entry); same results as rasterize_to_pixels_bwd."""
    return _raster_backward(means2d, conics, opacities, mus, None, tile_offsets, isect_ids, flatten_ids,
                            v_render_output, None, None, dim1, dim0, tile_size, absgrad, False)


def rasterize_to_pixels_mean_var_bwd_per_gaussian(means2d, conics, opacities, mus, tile_offsets, isect_ids,
                                                  flatten_ids, v_render_output, v_render_var, *args):
    """Joint VJP of mean and variance images.

    Two call forms, as the reference's overloads (ext.cpp:106-128):
    ``(..., v_render_var, dim1, dim0, tile_size, absgrad)`` -- detached variance branch;
    ``(..., v_render_var, uncertainties, detach, dim1, dim0, tile_size, absgrad)``.
    Returns (absgrad|None, v_means2d, v_conics, v_opacities, v_mus, v_uncertainties).
    """
    uncertainties, detach, dim1, dim0, tile_size, absgrad = _mean_var_args(args)
    unc = None if detach else uncertainties
    return _raster_backward(means2d, conics, opacities, mus, None, tile_offsets, isect_ids, flatten_ids,
                            v_render_output, v_render_var, unc, dim1, dim0, tile_size, absgrad, True)


def beta_rasterize_to_pixels_bwd(means2d, conics, opacities, mus, betas, tile_offsets, flatten_ids, v_render_output,
                                 dim1, dim0, tile_size, absgrad):
    """Beta image VJP: (absgrad|None, v_means2d, v_conics, v_opacities, v_mus, v_betas)."""
    return _raster_backward(means2d, conics, opacities, mus, betas, tile_offsets, None, flatten_ids, v_render_output,
                            None, None, dim1, dim0, tile_size, absgrad, False)


def beta_rasterize_to_pixels_bwd_per_gaussian(means2d, conics, opacities, mus, betas, tile_offsets, isect_ids,
                                              flatten_ids, v_render_output, dim1, dim0, tile_size, absgrad):
    return _raster_backward(means2d, conics, opacities, mus, betas, tile_offsets, isect_ids, flatten_ids,
                            v_render_output, None, None, dim1, dim0, tile_size, absgrad, False)


def beta_rasterize_to_pixels_mean_var_bwd_per_gaussian(means2d, conics, opacities, mus, betas, tile_offsets,
                                                       isect_ids, flatten_ids, v_render_output, v_render_var, *args):
    """Beta joint VJP; returns (..., v_mus, v_betas, v_uncertainties). Call forms as the Gaussian one."""
    uncertainties, detach, dim1, dim0, tile_size, absgrad = _mean_var_args(args)
    unc = None if detach else uncertainties
    return _raster_backward(means2d, conics, opacities, mus, betas, tile_offsets, isect_ids, flatten_ids,
                            v_render_output, v_render_var, unc, dim1, dim0, tile_size, absgrad, True)


def _mean_var_args(args):
    if len(args) == 4:
        dim1, dim0, tile_size, absgrad = args
        return None, True, dim1, dim0, tile_size, absgrad
    if len(args) == 6:
        uncertainties, detach, dim1, dim0, tile_size, absgrad = args
        return uncertainties, bool(detach), dim1, dim0, tile_size, absgrad
    raise TypeError("mean/variance VJP takes (dim1, dim0, tile_size, absgrad) or "
                    "(uncertainties, detach, dim1, dim0, tile_size, absgrad) after v_render_var")


# ---------------------------------------------------------------------------
# voxelization
# ---------------------------------------------------------------------------

def _voxel_inputs(means3d, conics, opacities, betas, tile_offsets, flatten_ids, isect_ids=None):
    _check("means3d", means3d)
    _dtype(means3d)
    _check_float("conics", conics, means3d)
    _check_float("opacities", opacities, means3d)
    _check("tile_offsets", tile_offsets, means3d.device)
    _check("flatten_ids", flatten_ids, means3d.device)
    _require(means3d.dim() == 2, "means3d must be 2D [N, 3]")
    _require(conics.dim() == 2, "conics must be 2D [N, 6]")
    _require(opacities.dim() == 1, "opacities must be 1D [N]")
    _require(tile_offsets.dim() == 3, "tile_offsets must be 3D [n_tiles_dim0, n_tiles_dim1, n_tiles_dim2]")
    _require(flatten_ids.dim() == 1, "flatten_ids must be 1D [n_isects]")
    n = means3d.size(0)
    _require(means3d.size(1) == 3 and conics.shape == (n, 6) and opacities.shape == (n,),
             "means3d [N,3], conics [N,6] and opacities [N] must agree")
    if betas is not None:
        _check_float("betas", betas, means3d)
        _require(betas.dim() == 1 and betas.size(0) == n, "betas must be 1D [N]")
    if isect_ids is not None:
        _check("isect_ids", isect_ids, means3d.device)
        _require(isect_ids.dim() == 1, "isect_ids must be 1D")
    tz, ty, tx = tile_offsets.shape
    return n, flatten_ids.size(0), tx, ty, tz


def _voxel_forward(means3d, conics, opacities, betas, uncertainties, tile_offsets, flatten_ids, dim2, dim1, dim0,
                   tile_size):
    n, m, tx, ty, tz = _voxel_inputs(means3d, conics, opacities, betas, tile_offsets, flatten_ids)
    if uncertainties is not None:
        _check_float("uncertainties", uncertainties, means3d)
        _require(uncertainties.dim() == 1 and uncertainties.size(0) == n, "uncertainties must be 1D [N]")
    device = means3d.device
    vol = means3d.new_empty((int(dim0), int(dim1), int(dim2)))
    vol_var = torch.empty_like(vol) if uncertainties is not None else None
    with _Guard(device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_voxel_workspace(_dtype(means3d), n, 0), device)
        if uncertainties is None:
            _backend.call("r2s_voxelize_to_voxels_fwd", _dtype(means3d), _ptr(means3d), _ptr(conics),
                          _ptr(opacities), _ptr(betas), _ptr(tile_offsets), _ptr(flatten_ids), n, m, int(dim2),
                          int(dim1), int(dim0), int(tile_size), tx, ty, tz, _ptr(vol), _ptr(ws), ws.numel(),
                          _stream(device))
            return vol
        _backend.call("r2s_voxelize_to_voxels_mean_var_fwd", _dtype(means3d), _ptr(means3d), _ptr(conics),
                      _ptr(opacities), _ptr(betas), _ptr(uncertainties), _ptr(tile_offsets), _ptr(flatten_ids), n, m,
                      int(dim2), int(dim1), int(dim0), int(tile_size), tx, ty, tz, _ptr(vol), _ptr(vol_var),
                      _ptr(ws), ws.numel(), _stream(device))
    return vol, vol_var


def _voxel_backward(means3d, conics, opacities, betas, tile_offsets, isect_ids, flatten_ids, v_vol, v_vol_var,
                    uncertainties, dim2, dim1, dim0, tile_size, with_unc):
    n, m, tx, ty, tz = _voxel_inputs(means3d, conics, opacities, betas, tile_offsets, flatten_ids, isect_ids)
    shape = (int(dim0), int(dim1), int(dim2))
    if v_vol is not None:
        _check_float("v_render_output", v_vol, means3d)
        _require(v_vol.dim() == 3, "v_render_output must be 3D [dim0, dim1, dim2]")
        _require(tuple(v_vol.shape) == shape, "v_render_output shape must be [dim0, dim1, dim2]")
    if v_vol_var is not None:
        _check_float("v_render_var", v_vol_var, means3d)
        _require(v_vol_var.dim() == 3, "v_render_var must be 3D [dim0, dim1, dim2]")
        _require(tuple(v_vol_var.shape) == shape, "v_render_var shape must be [dim0, dim1, dim2]")
    if uncertainties is not None:
        _check_float("uncertainties", uncertainties, means3d)
        _require(uncertainties.dim() == 1 and uncertainties.size(0) == n, "uncertainties must be 1D [N]")
    device = means3d.device
    v_means = torch.empty_like(means3d)
    v_conics = torch.empty_like(conics)
    v_opac = torch.empty_like(opacities)
    v_betas = torch.empty_like(betas) if betas is not None else None
    v_unc = torch.zeros_like(opacities) if with_unc else None
    with _Guard(device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_voxel_workspace(_dtype(means3d), n, 1), device)
        _backend.call("r2s_voxelize_to_voxels_bwd", _dtype(means3d), _ptr(means3d), _ptr(conics), _ptr(opacities),
                      _ptr(betas), _ptr(tile_offsets), _ptr(isect_ids), _ptr(flatten_ids), _ptr(v_vol),
                      _ptr(v_vol_var), _ptr(uncertainties), n, m, int(dim2), int(dim1), int(dim0), int(tile_size),
                      tx, ty, tz, _ptr(v_means), _ptr(v_conics), _ptr(v_opac), _ptr(v_betas), _ptr(v_unc), _ptr(ws),
                      ws.numel(), _stream(device))
    out = (v_means, v_conics, v_opac)
    if betas is not None:
        out += (v_betas,)
    if with_unc:
        out += (v_unc,)
    return out


def voxelize_to_voxels_fwd(means3d, conics, opacities, tile_offsets, flatten_ids, dim2, dim1, dim0, tile_size):
    """Gaussian densities at voxel centres -> volume [dim0, dim1, dim2]."""
    return _voxel_forward(means3d, conics, opacities, None, None, tile_offsets, flatten_ids, dim2, dim1, dim0,
                          tile_size)


def voxelize_to_voxels_mean_var_fwd(means3d, conics, opacities, uncertainties, tile_offsets, flatten_ids, dim2, dim1,
                                    dim0, tile_size):
    return _voxel_forward(means3d, conics, opacities, None, uncertainties, tile_offsets, flatten_ids, dim2, dim1,
                          dim0, tile_size)


def beta_voxelize_to_voxels_fwd(means3d, conics, opacities, betas, tile_offsets, flatten_ids, dim2, dim1, dim0,
                                tile_size):
    return _voxel_forward(means3d, conics, opacities, betas, None, tile_offsets, flatten_ids, dim2, dim1, dim0,
                          tile_size)


def beta_voxelize_to_voxels_mean_var_fwd(means3d, conics, opacities, betas, uncertainties, tile_offsets,
                                         flatten_ids, dim2, dim1, dim0, tile_size):
    return _voxel_forward(means3d, conics, opacities, betas, uncertainties, tile_offsets, flatten_ids, dim2, dim1,
                          dim0, tile_size)


def voxelize_to_voxels_bwd(means3d, conics, opacities, tile_offsets, flatten_ids, v_render_output, dim2, dim1, dim0,
                           tile_size):
    """Volume VJP ("pixel" mode entry): (v_means3d, v_conics, v_opacities)."""
    return _voxel_backward(means3d, conics, opacities, None, tile_offsets, None, flatten_ids, v_render_output, None,
                           None, dim2, dim1, dim0, tile_size, False)


def voxelize_to_voxels_bwd_per_gaussian(means3d, conics, opacities, tile_offsets, isect_ids, flatten_ids,
                                        v_render_output, dim2, dim1, dim0, tile_size):
    return _voxel_backward(means3d, conics, opacities, None, tile_offsets, isect_ids, flatten_ids, v_render_output,
                           None, None, dim2, dim1, dim0, tile_size, False)


def voxelize_to_voxels_mean_var_bwd_per_gaussian(means3d, conics, opacities, tile_offsets, isect_ids, flatten_ids,
                                                 v_render_output, v_render_var, *args):
    """Joint volume VJP; overloads as ext.cpp:42-63. -> (v_means3d, v_conics, v_opacities, v_uncertainties)."""
    uncertainties, detach, dim2, dim1, dim0, tile_size = _voxel_mean_var_args(args)
    return _voxel_backward(means3d, conics, opacities, None, tile_offsets, isect_ids, flatten_ids, v_render_output,
                           v_render_var, None if detach else uncertainties, dim2, dim1, dim0, tile_size, True)


def beta_voxelize_to_voxels_bwd(means3d, conics, opacities, betas, tile_offsets, flatten_ids, v_render_output, dim2,
                                dim1, dim0, tile_size):
    return _voxel_backward(means3d, conics, opacities, betas, tile_offsets, None, flatten_ids, v_render_output, None,
                           None, dim2, dim1, dim0, tile_size, False)


def beta_voxelize_to_voxels_bwd_per_gaussian(means3d, conics, opacities, betas, tile_offsets, isect_ids,
                                             flatten_ids, v_render_output, dim2, dim1, dim0, tile_size):
    return _voxel_backward(means3d, conics, opacities, betas, tile_offsets, isect_ids, flatten_ids, v_render_output,
                           None, None, dim2, dim1, dim0, tile_size, False)


def beta_voxelize_to_voxels_mean_var_bwd_per_gaussian(means3d, conics, opacities, betas, tile_offsets, isect_ids,
                                                      flatten_ids, v_render_output, v_render_var, *args):
    uncertainties, detach, dim2, dim1, dim0, tile_size = _voxel_mean_var_args(args)
    return _voxel_backward(means3d, conics, opacities, betas, tile_offsets, isect_ids, flatten_ids, v_render_output,
                           v_render_var, None if detach else uncertainties, dim2, dim1, dim0, tile_size, True)


def _voxel_mean_var_args(args):
    if len(args) == 4:
        dim2, dim1, dim0, tile_size = args
        return None, True, dim2, dim1, dim0, tile_size
    if len(args) == 6:
        uncertainties, detach, dim2, dim1, dim0, tile_size = args
        return uncertainties, bool(detach), dim2, dim1, dim0, tile_size
    raise TypeError("mean/variance VJP takes (dim2, dim1, dim0, tile_size) or "
                    "(uncertainties, detach, dim2, dim1, dim0, tile_size) after v_render_var")


# ---------------------------------------------------------------------------
# losses
# ---------------------------------------------------------------------------

def volume_loss_fwd(volume: Tensor, lambda_tv: float):
    """Anisotropic TV of a [B,D,H,W] volume -> (lambda * tv, tv, tv_map)."""
    _check("volume", volume)
    _dtype(volume)
    _require(volume.dim() == 4, "volume must be 4D (B, D, H, W)")
    b, d, h, w = volume.shape
    tv_map = torch.empty_like(volume)
    loss = volume.new_empty(())
    tv = volume.new_empty(())
    with _Guard(volume.device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_volume_loss_workspace(volume.numel()), volume.device)
        _backend.call("r2s_volume_loss_fwd", _dtype(volume), _ptr(volume), b, d, h, w, float(lambda_tv), _ptr(loss),
                      _ptr(tv), _ptr(tv_map), _ptr(ws), ws.numel(), _stream(volume.device))
    return loss, tv, tv_map


def volume_loss_bwd(volume: Tensor, grad_output: Tensor, lambda_tv: float):
    """Gradient of lambda * TV with respect to the volume, scaled by grad_output[0]."""
    _check("volume", volume)
    _check("grad_output", grad_output)
    _require(grad_output.device == volume.device, "grad_output must be on the same CUDA device as volume")
    _dtype(volume)
    _require(volume.dim() == 4, "volume must be 4D (B, D, H, W)")
    _require(grad_output.dtype == volume.dtype and grad_output.numel() >= 1, "grad_output must match volume's dtype")
    b, d, h, w = volume.shape
    grad = torch.empty_like(volume)
    if volume.numel():
        with _Guard(volume.device):
            _backend.call("r2s_volume_loss_bwd", _dtype(volume), _ptr(volume), _ptr(grad_output), b, d, h, w,
                          float(lambda_tv), _ptr(grad), _stream(volume.device))
    return grad


def volume_loss_fwd_bwd(volume: Tensor, grad_output: Tensor, lambda_tv: float, with_map: bool = False):
    """``volume_loss_fwd`` and ``volume_loss_bwd`` in one pass over the volume.

    No reference counterpart as one call: for a caller that knows the upstream
    gradient before the forward (a fit step, where the TV term enters the loss
    with weight one). Returns ``(lambda * tv, tv, grad_volume)``, plus
    ``tv_map`` when ``with_map``; the map and the gradient equal the two
    separate calls' bit for bit.
    """
    _check("volume", volume)
    _check("grad_output", grad_output)
    _require(grad_output.device == volume.device, "grad_output must be on the same CUDA device as volume")
    _dtype(volume)
    _require(volume.dim() == 4, "volume must be 4D (B, D, H, W)")
    _require(grad_output.dtype == volume.dtype and grad_output.numel() >= 1, "grad_output must match volume's dtype")
    b, d, h, w = volume.shape
    grad = torch.empty_like(volume)
    tv_map = torch.empty_like(volume) if with_map else None
    loss = volume.new_empty(())
    tv = volume.new_empty(())
    with _Guard(volume.device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_volume_loss_workspace(volume.numel()), volume.device)
        _backend.call("r2s_volume_loss_fwd_bwd", _dtype(volume), _ptr(volume), _ptr(grad_output), b, d, h, w,
                      float(lambda_tv), _ptr(loss), _ptr(tv), _ptr(tv_map), _ptr(grad), _ptr(ws), ws.numel(),
                      _stream(volume.device))
    return (loss, tv, grad) + ((tv_map,) if with_map else ())


def image_loss_l1_fwd(prediction: Tensor, target: Tensor, lambda_l1: float):
    """Mean L1 of [B,H,W] images -> (lambda * l1, l1, l1_map)."""
    _check("prediction", prediction)
    _check("target", target)
    _require(target.device == prediction.device, "target must be on the same CUDA device as prediction")
    _dtype(prediction)
    _require(prediction.dim() == 3, "prediction must be 3D (B, H, W)")
    _require(target.dim() == 3, "target must be 3D (B, H, W)")
    _require(prediction.shape == target.shape, "prediction and target must have same shape")
    b, h, w = prediction.shape
    l1_map = torch.empty_like(prediction)
    loss = prediction.new_empty(())
    l1 = prediction.new_empty(())
    with _Guard(prediction.device):
        lib = _backend.library()
        ws = _workspace(lib.r2s_volume_loss_workspace(prediction.numel()), prediction.device)
        _backend.call("r2s_image_loss_l1_fwd", _dtype(prediction), _ptr(prediction), _ptr(target), b, h, w,
                      float(lambda_l1), _ptr(loss), _ptr(l1), _ptr(l1_map), _ptr(ws), ws.numel(),
                      _stream(prediction.device))
    return loss, l1, l1_map


def image_loss_l1_bwd(prediction: Tensor, target: Tensor, grad_output: Tensor, lambda_l1: float):
    """Gradient of lambda * mean L1 with respect to the prediction."""
    _check("prediction", prediction)
    _check("target", target)
    _require(target.device == prediction.device, "target must be on the same CUDA device as prediction")
    _check("grad_output", grad_output)
    _require(grad_output.device == prediction.device, "grad_output must be on the same CUDA device as prediction")
    _dtype(prediction)
    _require(prediction.dim() == 3, "prediction must be 3D (B, H, W)")
    _require(target.dim() == 3, "target must be 3D (B, H, W)")
    _require(prediction.shape == target.shape, "prediction and target must have same shape")
    b, h, w = prediction.shape
    grad = torch.empty_like(prediction)
    if prediction.numel():
        with _Guard(prediction.device):
            _backend.call("r2s_image_loss_l1_bwd", _dtype(prediction), _ptr(prediction), _ptr(target),
                          _ptr(grad_output), b, h, w, float(lambda_l1), _ptr(grad), _stream(prediction.device))
    return grad


image_loss_fwd = image_loss_l1_fwd
image_loss_bwd = image_loss_l1_bwd


def is_cuda_extension_available() -> bool:
    return _backend.is_cuda_available()


__all__ = [
    "image_loss_fwd", "image_loss_bwd", "image_loss_l1_fwd", "image_loss_l1_bwd",
    "volume_loss_fwd", "volume_loss_bwd",
    "isect_tiles", "isect_offset_encode", "isect_tiles_3d", "isect_offset_encode_3d",
    "voxelize_to_voxels_fwd", "voxelize_to_voxels_mean_var_fwd", "voxelize_to_voxels_bwd",
    "voxelize_to_voxels_bwd_per_gaussian", "voxelize_to_voxels_mean_var_bwd_per_gaussian",
    "beta_voxelize_to_voxels_fwd", "beta_voxelize_to_voxels_mean_var_fwd", "beta_voxelize_to_voxels_bwd",
    "beta_voxelize_to_voxels_bwd_per_gaussian", "beta_voxelize_to_voxels_mean_var_bwd_per_gaussian",
    "rasterize_to_pixels_fwd", "rasterize_to_pixels_mean_var_fwd", "rasterize_to_pixels_uncertainty_bwd",
    "rasterize_to_pixels_bwd", "rasterize_to_pixels_bwd_per_gaussian", "rasterize_to_pixels_mean_var_bwd_per_gaussian",
    "beta_rasterize_to_pixels_fwd", "beta_rasterize_to_pixels_mean_var_fwd",
    "beta_rasterize_to_pixels_uncertainty_bwd", "beta_rasterize_to_pixels_bwd",
    "beta_rasterize_to_pixels_bwd_per_gaussian", "beta_rasterize_to_pixels_mean_var_bwd_per_gaussian",
    "conics_mu_fwd", "conics_mu_bwd", "world_to_image_projection_fwd", "world_to_image_projection_bwd",
    "parameter_transform_fwd", "parameter_transform_bwd", "world_to_volume_mapping_fwd",
    "world_to_volume_mapping_bwd", "is_cuda_extension_available",
]
