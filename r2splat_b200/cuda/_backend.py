"""Loader for the in-tree sm_100a library (``r2splat_b200/_lib/libr2splat_b200.so``).

The library is a plain C-ABI shared object (declared in ``include/r2splat_b200.h``)
bound here with ctypes. There is no CPU implementation: if the library is
missing or CUDA is unavailable, the first operator call raises RuntimeError,
as the reference's lazy extension loader does (``r2splat/cuda/_backend.py:16-59``).
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import torch

_LIB_PATH = Path(__file__).resolve().parent.parent / "_lib" / "libr2splat_b200.so"

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I32 = ctypes.c_int
I64 = ctypes.c_int64
F32 = ctypes.c_float
F64 = ctypes.c_double
SZ = ctypes.c_size_t

# name -> (restype, argtypes); must match include/r2splat_b200.h.
SIGNATURES: dict[str, tuple] = {
    "r2s_abi_version": (I32, []),
    "r2s_last_error": (ctypes.c_char_p, []),
    "r2s_fp32_peak_probe": (I32, [P, U32, U32, I32, P]),
    "r2s_sfu_peak_probe": (I32, [P, U32, U32, I32, P]),
    "r2s_launch_count": (U64, []),
    "r2s_check_values": (I32, [I32, P, U32, P, P]),
    "r2s_parameter_transform_fwd": (I32, [I32, P, P, P, P, U32, P]),
    "r2s_parameter_transform_bwd": (I32, [I32, P, P, P, P, P, U32, P]),
    "r2s_world_to_image_projection_fwd": (I32, [I32, P, P, P, P, U32, U32, U32, U32, F32, F32, P, P, P, P]),
    "r2s_world_to_image_projection_bwd": (I32, [I32, P, P, P, P, U32, U32, U32, U32, P, P, P, P, P]),
    "r2s_conics_mu_fwd": (I32, [I32, P, U32, F64, P, P, P]),
    "r2s_conics_mu_bwd": (I32, [I32, P, U32, F64, P, P, P, P, P, P]),
    "r2s_world_to_volume_mapping_fwd": (I32, [I32, P, P, P, P, U32, U32, U32, U32, F64, F64, P, P, P, P]),
    "r2s_world_to_volume_mapping_bwd": (I32, [I32, P, P, P, P, U32, U32, U32, U32, F64, P, P, P, P, P]),
    "r2s_isect_count_workspace": (SZ, [U64]),
    "r2s_isect_emit_workspace": (SZ, [U64, U64]),
    "r2s_scan_tile_counts": (I32, [P, U64, P, P, SZ, P]),
    "r2s_isect_tiles_count": (I32, [I32, P, P, I32, U32, U32, U32, U32, U32, P, P, P, SZ, P]),
    "r2s_isect_tiles_emit": (I32, [I32, P, P, I32, U32, U32, U32, U32, U32, P, I64, P, P, P, P, SZ, P]),
    "r2s_isect_offset_encode": (I32, [P, I64, U32, U32, U32, P, P]),
    "r2s_isect_tiles_3d_count": (I32, [I32, P, P, U32, U32, U32, U32, U32, P, P, P, SZ, P]),
    "r2s_isect_tiles_3d_emit": (I32, [I32, P, P, U32, U32, U32, U32, U32, P, I64, P, P, P, P, SZ, P]),
    "r2s_isect_offset_encode_3d": (I32, [P, I64, U32, U32, U32, P, P]),
    "r2s_raster_workspace": (SZ, [U32, U32, U32, I32]),
    "r2s_rasterize_to_pixels_fwd": (I32, [I32, P, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32, U32, U32,
                                          P, P, SZ, P]),
    "r2s_rasterize_to_pixels_mean_var_fwd": (I32, [I32, P, P, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32,
                                                   U32, U32, P, P, P, SZ, P]),
    "r2s_rasterize_to_pixels_uncertainty_bwd": (I32, [I32, P, P, P, P, P, P, P, P, U32, U32, U32, U32, U32,
                                                      U32, U32, U32, P, P, SZ, P]),
    "r2s_rasterize_to_pixels_bwd": (I32, [I32, P, P, P, P, P, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32,
                                          U32, U32, P, P, P, P, P, P, P, P, SZ, P]),
    "r2s_voxel_workspace": (SZ, [U32, U32, I32]),
    "r2s_voxelize_to_voxels_fwd": (I32, [I32, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32, U32, U32, U32,
                                         P, P, SZ, P]),
    "r2s_voxelize_to_voxels_mean_var_fwd": (I32, [I32, P, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32, U32,
                                                  U32, U32, P, P, P, SZ, P]),
    "r2s_voxelize_to_voxels_bwd": (I32, [I32, P, P, P, P, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32, U32,
                                         U32, U32, P, P, P, P, P, P, SZ, P]),
    "r2s_volume_loss_workspace": (SZ, [U64]),
    "r2s_volume_loss_fwd": (I32, [I32, P, U32, U32, U32, U32, F32, P, P, P, P, SZ, P]),
    "r2s_volume_loss_bwd": (I32, [I32, P, P, U32, U32, U32, U32, F32, P, P]),
    "r2s_volume_loss_fwd_bwd": (I32, [I32, P, P, U32, U32, U32, U32, F32, P, P, P, P, P, SZ, P]),
    "r2s_image_loss_l1_fwd": (I32, [I32, P, P, U32, U32, U32, F32, P, P, P, P, SZ, P]),
    "r2s_image_loss_l1_bwd": (I32, [I32, P, P, P, U32, U32, U32, F32, P, P]),
    "r2s_raster_project": (I32, [I32, P, P, P, P, P, P, P, U32, U32, U32, U32, F32, F64, F32, U32, U32, U32,
                                 P, P, P, P]),
    "r2s_raster_emit": (I32, [P, U32, U32, U32, U32, P, I64, P, P, P, P, SZ, P]),
    "r2s_raster_render": (I32, [I32, P, P, I32, P, P, U32, U32, U32, U32, U32, U32, U32, U32, P, P, P]),
    "r2s_raster_render_bwd": (I32, [I32, P, P, I32, I32, P, P, P, P, U32, U32, U32, U32, U32, U32, U32, U32,
                                    P, P, P, P]),
    "r2s_raster_record_bwd": (I32, [I32, P, P, P, I32, I32, P, P, U32, U32, U32, U32, U32, P, P, P, P]),
    "r2s_sum_over_cameras": (I32, [I32, P, U32, U32, P, P]),
    "r2s_raster_chain_bwd": (I32, [I32, P, P, P, P, P, P, P, P, P, U32, U32, U32, U32, F32, F64, P, P, P, P,
                                   P, P, P]),
    "r2s_voxel_project": (I32, [I32, P, P, P, P, P, P, P, U32, U32, U32, U32, F64, F64, U32, U32, U32, U32,
                                P, P, P, P, P]),
    "r2s_voxel_render": (I32, [I32, P, I32, P, P, U32, U32, U32, U32, U32, U32, U32, U32, U32, P, P, P]),
    "r2s_voxel_render_bwd": (I32, [I32, P, I32, I32, P, P, P, P, U32, U32, U32, U32, U32, U32, U32, U32, U32,
                                   P, P]),
    "r2s_voxel_chain_bwd": (I32, [I32, P, P, P, P, P, P, U32, U32, U32, U32, F64, P, P, P, P, P, P, P, P]),
    "r2s_raster_emit_capacity": (I32, [P, U32, U32, U32, U32, P, I64, P, P, P, P, P, P, SZ, P]),
    "r2s_voxel_emit_capacity": (I32, [I32, P, P, U32, U32, U32, U32, U32, P, I64, P, P, P, P, P, P, SZ, P]),
    "r2s_raster_render_capacity": (I32, [I32, P, P, I32, P, P, P, U32, U32, U32, U32, U32, U32, U32, U32, P, P,
                                         P]),
    "r2s_voxel_render_capacity": (I32, [I32, P, I32, P, P, P, U32, U32, U32, U32, U32, U32, U32, U32, P, P, P]),
    "r2s_voxel_render_bwd_capacity": (I32, [I32, P, I32, I32, P, P, P, P, P, U32, U32, U32, U32, U32, U32, U32,
                                            U32, P, P]),
    # dtype, records, beta, detach, offsets, ids, n_isects, n_used, means_v, radii, tile_cum, v_volume, v_volume_var,
    # N, dim2, dim1, dim0, tile, tiles_x, tiles_y, tiles_z, slots, slot_capacity, grads, stream
    "r2s_voxel_render_bwd_slots": (I32, [I32, P, I32, I32, P, P, U64, P, P, P, P, P, P, U32, U32, U32, U32, U32, U32,
                                         U32, U32, P, U64, P, P]),
    "r2s_voxel_pack_workspace": (SZ, [U32]),
    # dtype, records, offsets, flatten_ids, radii, tile_cum, N, n_isects, n_used, tile, tiles_x, tiles_y, tiles_z,
    # slot_capacity, packed, workspace, bytes, stream
    "r2s_voxel_pack_tile_records": (I32, [I32, P, P, P, P, P, U32, U64, P, U32, U32, U32, U32, U64, P, P, SZ, P]),
    # dtype, packed, beta, offsets, n_isects, n_used, dim2, dim1, dim0, tile, tiles_x, tiles_y, tiles_z, volume,
    # volume_var, stream
    "r2s_voxel_render_packed": (I32, [I32, P, I32, P, U64, P, U32, U32, U32, U32, U32, U32, U32, P, P, P]),
    # dtype, packed, beta, detach, offsets, n_isects, n_used, tile_cum, v_volume, v_volume_var, N, dim2, dim1, dim0,
    # tile, tiles_x, tiles_y, tiles_z, slots, slot_capacity, grads, stream
    "r2s_voxel_render_bwd_packed": (I32, [I32, P, I32, I32, P, U64, P, P, P, P, U32, U32, U32, U32, U32, U32, U32,
                                          U32, P, U64, P, P]),
    "r2s_bulk_wait_faults": (I32, [I32, I32, P]),
    "r2s_voxel_layer_counts": (I32, [I32, P, P, U32, U32, U32, U32, U32, U32, U32, U32, P, P]),
    # dtype, records, means_v, radii, layer_cum, n_items, n_items_dev, beta, detach, v_volume, v_volume_var, N,
    # dim2, dim1, dim0, tile, tiles_x, tiles_y, tiles_z, partials, grads, overflow, stream
    "r2s_voxel_record_bwd": (I32, [I32, P, P, P, P, U64, P, I32, I32, P, P, U32, U32, U32, U32, U32, U32, U32, U32,
                                   P, P, P, P]),
    "r2s_raster_image_loss_workspace": (SZ, [U32, U32, U32]),
    # dtype, records, unc, beta, offsets, ids, n_isects, n_used, C, N, W, H, tile, tiles_x, tiles_y, stage_batch,
    # target, kind, lambda, render, render_var, v_render, loss, loss_value, workspace, bytes, stream
    "r2s_raster_render_image_loss": (I32, [I32, P, P, I32, P, P, U32, P, U32, U32, U32, U32, U32, U32, U32, U32,
                                           P, I32, F32, P, P, P, P, P, P, SZ, P]),
    "r2s_adam_activation_step": (I32, [I32, U32, P, P, P, P, P, P, P, P, P, P, P, P, F64, F64, F64, F64, P, P, P]),
    "r2s_scan_tile_counts_noalloc_max": (U64, []),
    "r2s_scan_tile_counts_noalloc": (I32, [P, U64, P, P]),
}

_lock = threading.Lock()
_lib = None
_load_error: str | None = None


def library_path() -> Path:
    return _LIB_PATH


def _load():
    global _lib, _load_error
    with _lock:
        if _lib is not None or _load_error is not None:
            return _lib
        if not _LIB_PATH.exists():
            _load_error = (f"r2splat_b200 CUDA library not found at {_LIB_PATH}; build it with "
                           "`python -m r2splat_b200.build`")
            return None
        try:
            lib = ctypes.CDLL(str(_LIB_PATH))
        except OSError as error:
            _load_error = f"failed to load {_LIB_PATH}: {error}"
            return None
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return _lib


def library():
    """The loaded ctypes library; raises RuntimeError when unavailable."""
    lib = _load()
    if lib is None:
        raise RuntimeError(_load_error)
    return lib


def is_library_loadable() -> bool:
    return _load() is not None


def is_cuda_available() -> bool:
    return torch.cuda.is_available() and is_library_loadable()


def call(name: str, *args) -> None:
    """Calls a C entry point and converts a nonzero status to RuntimeError."""
    lib = library()
    if not torch.cuda.is_available():
        raise RuntimeError("r2splat_b200 operators require a CUDA device")
    status = getattr(lib, name)(*args)
    if status != 0:
        message = lib.r2s_last_error().decode(errors="replace")
        raise RuntimeError(f"{name[4:]}: {message}")


__all__ = ["SIGNATURES", "call", "is_cuda_available", "is_library_loadable", "library", "library_path"]
