"""Fused device pipelines behind the explicit operators.

Rasterize (the reference's explicit.py:160-183 and :204-241):
  parameter transform -> one fused projection/conic/packing pass writing 32-byte
  records [C,N,8] + tile rectangles + tile counts -> int64 prefix sum -> host
  read of the intersection count -> emission + stable radix sort + per-tile
  offsets -> tile accumulation. The VJP needs no tile order: one warp per
  (camera, primitive) record walks the pixels of the record's tile rectangle
  and writes its packed adjoints [C,N,8] once, then one per-primitive
  chain-rule pass (conic/mu VJP, projection VJP summed over cameras, Beta path
  factor, parameter-transform VJP); neither uses atomics.

Voxelize (explicit.py:286-307, :331-350): the same structure in 3D with
64-byte records [N,16]. Its VJP is tile-parallel over the sorted lists, but
deterministic: each (tile, primitive) pair writes its sums to a slot of its
own and one pass adds each primitive's slots in a fixed order, so the voxel
gradients, like the raster ones, are the same on every run. A backward that
keeps no lists (recompute under a memory budget) walks each primitive's tile
box layer by layer instead (record-parallel, also deterministic).

All arrays are allocated through the torch caching allocator and passed to the
C ABI; nothing here computes on the CPU.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import torch

from . import _beta
from .cuda import _backend
from .cuda import _wrapper as low

Tensor = torch.Tensor
RASTER_TILE = 16
VOXEL_TILE = 8
# Largest scratch the deterministic voxel VJP takes for its per-intersection slots (12 values each);
# past it the VJP walks the primitives' tile boxes instead (one slot per primitive and z-layer).
VOXEL_SLOT_BUDGET_BYTES = 8 << 30
# The voxel forward copies the 3D records into per-tile packed order (16 values per intersection) when
# that copy and the VJP's slots fit this budget together; otherwise the tile kernels gather the records
# through the lists, as the reference's do.
VOXEL_PACK_BUDGET_BYTES = VOXEL_SLOT_BUDGET_BYTES


def _ptr(t: Optional[Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _dtype(t: Tensor) -> int:
    return 0 if t.dtype == torch.float32 else 1


def _ws(nbytes: int, device) -> Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


class StageTimer:
    """Optional CUDA-event timing of the pipeline stages (used by the benchmark).

    While ``active`` holds a StageTimer, each named stage records a start/end
    event pair on the current stream; ``totals_ms()`` sums them per stage after
    a synchronize.
    """

    active: "Optional[StageTimer]" = None

    def __init__(self):
        self.records: list[tuple[str, torch.cuda.Event, torch.cuda.Event]] = []

    def totals_ms(self) -> dict:
        out: dict = {}
        for name, start, end in self.records:
            out[name] = out.get(name, 0.0) + start.elapsed_time(end)
        return out


class _stage:
    """A named pipeline stage: an NVTX range (visible to nsys / ncu --nvtx) and, while a StageTimer is
    active, a CUDA-event pair."""

    def __init__(self, name: str):
        self.name = name
        self.start = None

    def __enter__(self):
        torch.cuda.nvtx.range_push("r2s:" + self.name)
        if StageTimer.active is not None:
            self.start = torch.cuda.Event(enable_timing=True)
            self.start.record()
        return self

    def __exit__(self, *exc):
        if self.start is not None and StageTimer.active is not None:
            end = torch.cuda.Event(enable_timing=True)
            end.record()
            StageTimer.active.records.append((self.name, self.start, end))
        torch.cuda.nvtx.range_pop()
        return False


@dataclass
class RasterState:
    """Device buffers a projection VJP needs (the reference saves 12, explicit.py:184-186)."""

    covars: Tensor
    records: Tensor
    offsets: Tensor
    isect_ids: Tensor
    flatten_ids: Tensor
    ratio: Optional[Tensor]
    n_isects: int
    width: int
    height: int
    tile_size: int = RASTER_TILE
    extra: dict = field(default_factory=dict)


@dataclass
class VoxelState:
    """Device buffers of a voxelize forward. The VJP reads the records, the voxel-space
    means and radii (its tile boxes) and the inclusive scan of the per-primitive layer
    counts; the sorted lists serve the forward (and callers that inspect them)."""

    covars: Tensor
    records: Tensor
    offsets: Optional[Tensor]
    isect_ids: Optional[Tensor]
    flatten_ids: Optional[Tensor]
    n_isects: int
    shape: tuple
    tile_size: int = VOXEL_TILE
    means_v: Optional[Tensor] = None
    radii: Optional[Tensor] = None
    tile_cum: Optional[Tensor] = None
    layer_cum: Optional[Tensor] = None
    n_items: int = 0
    packed: Optional[Tensor] = None  # per-tile packed records [M,16], the VJP slot in each padding


def raster_intersections(means, covars, densities, beta, ratio, viewmats, Ks, width, height, eps, radius_clip,
                         tile_size=RASTER_TILE, before_count=None):
    """Projection + packing + sorted tile intersections.

    Returns (records, offsets, isect_ids, flatten_ids, M, rects); rects [C,N,4] are the tile rectangles.
    ``before_count`` runs just before the host reads the intersection count (the pending input checks).
    """
    device = means.device
    c, n = viewmats.shape[0], means.shape[0]
    tx = (width + tile_size - 1) // tile_size
    ty = (height + tile_size - 1) // tile_size
    stream = _stream(device)
    lib = _backend.library()
    records = means.new_empty((c, n, 8))
    rects = torch.empty((c, n, 4), dtype=torch.int16, device=device)
    counts = torch.empty((c, n), dtype=torch.int32, device=device)
    _backend.call("r2s_raster_project", _dtype(means), _ptr(means), _ptr(covars), _ptr(densities), _ptr(beta),
                  _ptr(ratio), _ptr(viewmats), _ptr(Ks), c, n, width, height, float(eps), float(eps),
                  float(radius_clip), tile_size, tx, ty, _ptr(records), _ptr(rects), _ptr(counts), stream)
    cum = torch.empty((c * n,), dtype=torch.int64, device=device)
    ws = _ws(lib.r2s_isect_count_workspace(c * n), device)
    _backend.call("r2s_scan_tile_counts", _ptr(counts), c * n, _ptr(cum), _ptr(ws), ws.numel(), stream)
    if before_count is not None:
        before_count()
    m = int(cum[-1].item())
    isect_ids = torch.empty((m,), dtype=torch.int64, device=device)
    flatten_ids = torch.empty((m,), dtype=torch.int32, device=device)
    offsets = torch.empty((c, ty, tx), dtype=torch.int32, device=device)
    ws = _ws(lib.r2s_isect_emit_workspace(m, c * tx * ty), device)
    with _stage("raster_sort"):
        _backend.call("r2s_raster_emit", _ptr(rects), c, n, tx, ty, _ptr(cum), m, _ptr(isect_ids),
                      _ptr(flatten_ids), _ptr(offsets), _ptr(ws), ws.numel(), stream)
    return records, offsets, isect_ids, flatten_ids, m, rects


IMAGE_LOSS_KINDS = {"mse": 0, "l1": 1}  # R2S_IMAGE_LOSS_MSE, R2S_IMAGE_LOSS_L1


def render_image_loss(records, uncertainty, beta: bool, offsets, flatten_ids, m, n, width, height, tile_size,
                      target, kind, weight, image, variance, device):
    """Tile forward with the fused image-loss epilogue; returns (v_image, loss, loss_value).

    ``records`` and ``flatten_ids`` may be None when ``m`` is 0 (no
    intersections): the epilogue then sees an all-zero image.
    """
    c = target.shape[0]
    tx = (width + tile_size - 1) // tile_size
    ty = (height + tile_size - 1) // tile_size
    lib = _backend.library()
    ws = _ws(int(lib.r2s_raster_image_loss_workspace(c, tx, ty)), device)
    v_image = torch.empty_like(target)
    loss = target.new_empty(())
    value = target.new_empty(())
    _backend.call("r2s_raster_render_image_loss", _dtype(target), _ptr(records), _ptr(uncertainty), int(beta),
                  _ptr(offsets), _ptr(flatten_ids), m, None, c, n, width, height, tile_size, tx, ty, 0,
                  _ptr(target), IMAGE_LOSS_KINDS[kind], float(weight), _ptr(image), _ptr(variance), _ptr(v_image),
                  _ptr(loss), _ptr(value), _ptr(ws), ws.numel(), _stream(device))
    return v_image, loss, value


def raster_forward(means, quats, scales, densities, viewmats, Ks, width, height, beta, uncertainty, eps,
                   radius_clip, tile_size=RASTER_TILE, image_loss=None, before_count=None):
    """Explicit projection forward; returns (image or (image, variance), RasterState).

    With ``image_loss = (target, kind, weight)`` the tile kernel also writes the
    loss gradient; the return is then (output, state, (v_image, loss, loss_value)).
    """
    device = means.device
    c = viewmats.shape[0]
    covars, _ = low.parameter_transform_fwd(quats, scales)
    ratio = _beta.beta_path_ratio(beta) if beta is not None else None
    records, offsets, isect_ids, flatten_ids, m, rects = raster_intersections(
        means, covars, densities, beta, ratio, viewmats, Ks, width, height, eps, radius_clip, tile_size,
        before_count)
    image = means.new_empty((c, height, width))
    variance = torch.empty_like(image) if uncertainty is not None else None
    tx = (width + tile_size - 1) // tile_size
    ty = (height + tile_size - 1) // tile_size
    loss_out = None
    with _stage("raster_render"):
        if image_loss is None:
            _backend.call("r2s_raster_render", _dtype(means), _ptr(records), _ptr(uncertainty),
                          int(beta is not None), _ptr(offsets), _ptr(flatten_ids), c, means.shape[0], m, width,
                          height, tile_size, tx, ty, _ptr(image), _ptr(variance), _stream(device))
        else:
            target, kind, weight = image_loss
            loss_out = render_image_loss(records, uncertainty, beta is not None, offsets, flatten_ids, m,
                                         means.shape[0], width, height, tile_size, target, kind, weight, image,
                                         variance, device)
    state = RasterState(covars, records, offsets, isect_ids, flatten_ids, ratio, m, width, height, tile_size,
                        extra={"rects": rects})
    output = image if uncertainty is None else (image, variance)
    if image_loss is None:
        return output, state
    return output, state, loss_out


def raster_vjp_state(means, quats, scales, densities, viewmats, Ks, width, height, beta, eps, radius_clip,
                     tile_size=RASTER_TILE):
    """What the raster VJP reads (covariances, packed records, tile rectangles), rebuilt without the image.

    The record-parallel VJP needs neither the intersection lists nor their
    order, so recomputation is the parameter transform and the projection only.
    """
    device = means.device
    c, n = viewmats.shape[0], means.shape[0]
    tx = (width + tile_size - 1) // tile_size
    ty = (height + tile_size - 1) // tile_size
    covars, _ = low.parameter_transform_fwd(quats, scales)
    ratio = _beta.beta_path_ratio(beta) if beta is not None else None
    records = means.new_empty((c, n, 8))
    rects = torch.empty((c, n, 4), dtype=torch.int16, device=device)
    counts = torch.empty((c, n), dtype=torch.int32, device=device)
    _backend.call("r2s_raster_project", _dtype(means), _ptr(means), _ptr(covars), _ptr(densities), _ptr(beta),
                  _ptr(ratio), _ptr(viewmats), _ptr(Ks), c, n, width, height, float(eps), float(eps),
                  float(radius_clip), tile_size, tx, ty, _ptr(records), _ptr(rects), _ptr(counts), _stream(device))
    return RasterState(covars, records, None, None, None, ratio, 0, width, height, tile_size, extra={"rects": rects})


def voxel_vjp_state(means, quats, scales, densities, shape, extent, center, beta, uncertainty, eps, radius_clip,
                    tile_size=VOXEL_TILE):
    """What the voxel VJP reads (covariances, records, voxel-space means and radii, layer scan),
    rebuilt without the volume: the projection and the layer counts, no intersection lists or sort."""
    covars, _ = low.parameter_transform_fwd(quats, scales)
    records, means_v, radii, _, _ = _voxel_project(means, covars, densities, beta, uncertainty, extent, center,
                                                   shape, eps, radius_clip, tile_size)
    layer_cum = _layer_scan(means_v, radii, shape, tile_size)
    n_items = int(layer_cum[-1].item()) if layer_cum.numel() else 0
    return VoxelState(covars, records, None, None, None, 0, tuple(shape), tile_size, means_v, radii, None,
                      layer_cum, n_items)


def raster_backward(state: RasterState, means, quats, scales, densities, beta, uncertainty, viewmats, Ks, eps,
                    v_image, v_variance, detach_variance):
    """Explicit projection VJP -> (v_means, v_quats, v_scales, v_densities, v_beta, v_uncertainty)."""
    device = means.device
    c, n = viewmats.shape[0], means.shape[0]
    tile = state.tile_size
    stream = _stream(device)
    grads = means.new_empty((c, n, 8))  # every record is written by the record-parallel VJP
    # With the variance branch: one uncertainty adjoint per record, summed over cameras in order.
    v_unc_cn = means.new_empty((c, n)) if v_variance is not None else None
    v_unc = means.new_empty((n,)) if v_variance is not None else None
    with _stage("raster_render_bwd"):
        _backend.call("r2s_raster_record_bwd", _dtype(means), _ptr(state.records), _ptr(state.extra["rects"]),
                      _ptr(uncertainty), int(beta is not None), int(bool(detach_variance)), _ptr(v_image),
                      _ptr(v_variance), c, n, state.width, state.height, tile, _ptr(grads), None, _ptr(v_unc_cn),
                      stream)
    if v_unc is not None:
        _backend.call("r2s_sum_over_cameras", _dtype(means), _ptr(v_unc_cn), c, n, _ptr(v_unc), stream)
    log_grad = _beta.beta_path_log_grad(beta) if beta is not None else None
    v_means = means.new_empty((n, 3))
    v_quats = means.new_empty((n, 4))
    v_scales = means.new_empty((n, 3))
    v_dens = means.new_empty((n,))
    v_beta = means.new_empty((n,)) if beta is not None else None
    _backend.call("r2s_raster_chain_bwd", _dtype(means), _ptr(means), _ptr(quats), _ptr(scales), _ptr(state.covars),
                  _ptr(beta), _ptr(state.ratio), _ptr(log_grad), _ptr(viewmats), _ptr(Ks), c, n, state.width,
                  state.height, float(eps), float(eps), _ptr(grads), _ptr(v_means), _ptr(v_quats), _ptr(v_scales),
                  _ptr(v_dens), _ptr(v_beta), stream)
    if v_unc is None and uncertainty is not None:
        v_unc = torch.zeros_like(uncertainty)
    return v_means, v_quats, v_scales, v_dens, v_beta, v_unc


def _voxel_tiles(shape, tile_size):
    depth, height, width = shape
    return (width + tile_size - 1) // tile_size, (height + tile_size - 1) // tile_size, \
        (depth + tile_size - 1) // tile_size


def _voxel_project(means, covars, densities, beta, uncertainty, extent, center, shape, eps, radius_clip, tile_size):
    """Records [N,16], voxel-space means, radii, tile counts and their inclusive scan."""
    device = means.device
    depth, height, width = shape
    n = means.shape[0]
    tx, ty, tz = _voxel_tiles(shape, tile_size)
    stream = _stream(device)
    lib = _backend.library()
    records = means.new_empty((n, 16))
    means_v = means.new_empty((n, 3))
    radii = torch.empty((n, 3), dtype=torch.int32, device=device)
    counts = torch.empty((n,), dtype=torch.int32, device=device)
    _backend.call("r2s_voxel_project", _dtype(means), _ptr(means), _ptr(covars), _ptr(densities), _ptr(beta),
                  _ptr(uncertainty), _ptr(extent), _ptr(center), n, width, height, depth, float(eps),
                  float(radius_clip), tile_size, tx, ty, tz, _ptr(records), _ptr(means_v), _ptr(radii), _ptr(counts),
                  stream)
    cum = torch.empty((n,), dtype=torch.int64, device=device)
    ws = _ws(lib.r2s_isect_count_workspace(n), device)
    _backend.call("r2s_scan_tile_counts", _ptr(counts), n, _ptr(cum), _ptr(ws), ws.numel(), stream)
    return records, means_v, radii, counts, cum


def _layer_scan(means_v, radii, shape, tile_size):
    """Inclusive scan of the per-primitive z-layer counts of the 3D tile boxes (the VJP's work items)."""
    device = means_v.device
    depth, height, width = shape
    n = means_v.shape[0]
    tx, ty, tz = _voxel_tiles(shape, tile_size)
    stream = _stream(device)
    layers = torch.empty((n,), dtype=torch.int32, device=device)
    _backend.call("r2s_voxel_layer_counts", _dtype(means_v), _ptr(means_v), _ptr(radii), n, width, height, depth,
                  tile_size, tx, ty, tz, _ptr(layers), stream)
    layer_cum = torch.empty((n,), dtype=torch.int64, device=device)
    ws = _ws(_backend.library().r2s_isect_count_workspace(n), device)
    _backend.call("r2s_scan_tile_counts", _ptr(layers), n, _ptr(layer_cum), _ptr(ws), ws.numel(), stream)
    return layer_cum


def voxel_intersections(means, covars, densities, beta, uncertainty, extent, center, shape, eps, radius_clip,
                        tile_size=VOXEL_TILE, before_count=None):
    """Projection and sorted 3D tile lists.

    Returns (records, offsets, isect_ids, flatten_ids, M, means_v, radii, tile_cum); tile_cum is the
    inclusive scan of the per-primitive tile counts, which the VJP's slots are numbered by.
    """
    device = means.device
    tx, ty, tz = _voxel_tiles(shape, tile_size)
    stream = _stream(device)
    lib = _backend.library()
    records, means_v, radii, _, cum = _voxel_project(means, covars, densities, beta, uncertainty, extent, center,
                                                     shape, eps, radius_clip, tile_size)
    if before_count is not None:
        before_count()
    m = int(cum[-1].item())
    isect_ids = torch.empty((m,), dtype=torch.int64, device=device)
    flatten_ids = torch.empty((m,), dtype=torch.int32, device=device)
    offsets = torch.empty((tz, ty, tx), dtype=torch.int32, device=device)
    ws = _ws(lib.r2s_isect_emit_workspace(m, tx * ty * tz), device)
    with _stage("voxel_sort"):
        _backend.call("r2s_isect_tiles_3d_emit", _dtype(means), _ptr(means_v), _ptr(radii), means.shape[0],
                      tile_size, tx, ty, tz, _ptr(cum), m, _ptr(isect_ids), _ptr(flatten_ids), _ptr(offsets),
                      _ptr(ws), ws.numel(), stream)
    return records, offsets, isect_ids, flatten_ids, m, means_v, radii, cum


def release_lists(state):
    """Drops a forward state's intersection lists (raster or voxel): neither VJP needs them (the raster VJP
    walks tile rectangles; the voxel VJP then takes its list-free form), so a caller short of memory can
    free them between forward and backward. Returns the tensors dropped."""
    dropped = [t for t in (state.isect_ids, state.flatten_ids, state.offsets, getattr(state, "packed", None))
               if t is not None]
    state.isect_ids = state.flatten_ids = state.offsets = None
    if hasattr(state, "packed"):
        state.packed = None
    return dropped


def pack_tile_records(records, offsets, flatten_ids, radii, tile_cum, m, shape, tile_size):
    """Per-tile packed copy of the 3D records ([M,16], the sorted intersections' records in list order, each
    pair's VJP slot in the padding): each tile's batch is then one contiguous range, staged by one bulk copy."""
    tx, ty, tz = _voxel_tiles(shape, tile_size)
    n = records.shape[0]
    packed = records.new_empty((max(m, 1), records.shape[1]))
    ws = _ws(_backend.library().r2s_voxel_pack_workspace(n), records.device)
    _backend.call("r2s_voxel_pack_tile_records", _dtype(records), _ptr(records), _ptr(offsets), _ptr(flatten_ids),
                  _ptr(radii), _ptr(tile_cum), n, m, None, tile_size, tx, ty, tz, m, _ptr(packed), _ptr(ws),
                  ws.numel(), _stream(records.device))
    return packed


def voxel_forward(means, quats, scales, densities, shape, extent, center, beta, uncertainty, eps, radius_clip,
                  tile_size=VOXEL_TILE, before_count=None):
    device = means.device
    depth, height, width = shape
    covars, _ = low.parameter_transform_fwd(quats, scales)
    records, offsets, isect_ids, flatten_ids, m, means_v, radii, tile_cum = voxel_intersections(
        means, covars, densities, beta, uncertainty, extent, center, shape, eps, radius_clip, tile_size,
        before_count)
    volume = means.new_empty(shape)
    variance = torch.empty_like(volume) if uncertainty is not None else None
    tx = (width + tile_size - 1) // tile_size
    ty = (height + tile_size - 1) // tile_size
    tz = (depth + tile_size - 1) // tile_size
    packed = None
    if m * (16 + 12) * means.element_size() <= VOXEL_PACK_BUDGET_BYTES:
        with _stage("voxel_pack"):
            packed = pack_tile_records(records, offsets, flatten_ids, radii, tile_cum, m, shape, tile_size)
    with _stage("voxel_render"):
        if packed is not None:
            _backend.call("r2s_voxel_render_packed", _dtype(means), _ptr(packed), int(beta is not None),
                          _ptr(offsets), m, None, width, height, depth, tile_size, tx, ty, tz, _ptr(volume),
                          _ptr(variance), _stream(device))
        else:
            _backend.call("r2s_voxel_render", _dtype(means), _ptr(records), int(beta is not None), _ptr(offsets),
                          _ptr(flatten_ids), means.shape[0], m, width, height, depth, tile_size, tx, ty, tz,
                          _ptr(volume), _ptr(variance), _stream(device))
    state = VoxelState(covars, records, offsets, isect_ids, flatten_ids, m, tuple(shape), tile_size, means_v, radii,
                       tile_cum, packed=packed)
    return (volume if uncertainty is None else (volume, variance)), state


def voxel_backward(state: VoxelState, means, quats, scales, beta, uncertainty, extent, center, eps, v_volume,
                   v_variance, detach_variance):
    """Explicit voxel VJP -> (v_means, v_quats, v_scales, v_densities, v_beta, v_uncertainty)."""
    device = means.device
    n = means.shape[0]
    depth, height, width = state.shape
    tile = state.tile_size
    tx, ty, tz = _voxel_tiles(state.shape, tile)
    stream = _stream(device)
    grads = means.new_empty((n, 16))  # every primitive's entry is written
    # The list-free form when no lists were kept, or when per-intersection slots would take more memory
    # than the budget (it needs one slot per primitive and tile-box z-layer instead).
    slot_bytes = state.n_isects * 12 * means.element_size()
    list_free = state.offsets is None or slot_bytes > VOXEL_SLOT_BUDGET_BYTES
    if list_free and state.layer_cum is None:
        state.layer_cum = _layer_scan(state.means_v, state.radii, state.shape, state.tile_size)
        state.n_items = int(state.layer_cum[-1].item()) if n else 0
    with _stage("voxel_render_bwd"):
        if not list_free:
            # Tile-parallel over the forward's sorted lists, one slot per (tile, primitive) pair.
            slots = means.new_empty((max(state.n_isects, 1), 12))
            if state.packed is not None:
                _backend.call("r2s_voxel_render_bwd_packed", _dtype(means), _ptr(state.packed),
                              int(beta is not None), int(bool(detach_variance)), _ptr(state.offsets),
                              state.n_isects, None, _ptr(state.tile_cum), _ptr(v_volume), _ptr(v_variance), n,
                              width, height, depth, tile, tx, ty, tz, _ptr(slots), slots.shape[0], _ptr(grads),
                              stream)
            else:
                _backend.call("r2s_voxel_render_bwd_slots", _dtype(means), _ptr(state.records),
                              int(beta is not None), int(bool(detach_variance)), _ptr(state.offsets),
                              _ptr(state.flatten_ids), state.n_isects, None, _ptr(state.means_v), _ptr(state.radii),
                              _ptr(state.tile_cum), _ptr(v_volume), _ptr(v_variance), n, width, height, depth,
                              tile, tx, ty, tz, _ptr(slots), slots.shape[0], _ptr(grads), stream)
        else:
            # No lists kept: record-parallel over the primitives' tile-box layers.
            partials = means.new_empty((max(state.n_items, 1), 16))
            _backend.call("r2s_voxel_record_bwd", _dtype(means), _ptr(state.records), _ptr(state.means_v),
                          _ptr(state.radii), _ptr(state.layer_cum), state.n_items, None, int(beta is not None),
                          int(bool(detach_variance)), _ptr(v_volume), _ptr(v_variance), n, width, height, depth,
                          tile, tx, ty, tz, _ptr(partials), _ptr(grads), None, stream)
    v_means = means.new_empty((n, 3))
    v_quats = means.new_empty((n, 4))
    v_scales = means.new_empty((n, 3))
    v_dens = means.new_empty((n,))
    v_beta = means.new_empty((n,)) if beta is not None else None
    v_unc = means.new_empty((n,)) if v_variance is not None else None
    _backend.call("r2s_voxel_chain_bwd", _dtype(means), _ptr(means), _ptr(quats), _ptr(scales), _ptr(state.covars),
                  _ptr(extent), _ptr(center), n, width, height, depth, float(eps), _ptr(grads), _ptr(v_means),
                  _ptr(v_quats), _ptr(v_scales), _ptr(v_dens), _ptr(v_beta), _ptr(v_unc), stream)
    if v_unc is None and uncertainty is not None:
        v_unc = torch.zeros_like(uncertainty)
    return v_means, v_quats, v_scales, v_dens, v_beta, v_unc
