"""Host-side contract tests: public surface, validation, C-ABI exports (no GPU)."""

import ctypes
import math
import re
from pathlib import Path

import pytest
import torch

import r2splat_b200
from r2splat_b200 import rasterize_fwd, voxelize_fwd
from r2splat_b200._validation import _options, _shape
from r2splat_b200.cuda import _backend

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "r2splat_b200.h"

LOW_LEVEL = {
    "image_loss_fwd", "image_loss_bwd", "image_loss_l1_fwd", "image_loss_l1_bwd", "volume_loss_fwd",
    "volume_loss_bwd", "isect_tiles", "isect_offset_encode", "isect_tiles_3d", "isect_offset_encode_3d",
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
}


def header_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for match in re.finditer(r"^\s*[a-z_][a-z0-9_ ]*?\**\s*(r2s_\w+)\s*\(([^;]*?)\)\s*;", text, flags=re.M):
        args = match.group(2).strip()
        out[match.group(1)] = 0 if args in ("", "void") else args.count(",") + 1
    return out


def test_public_api_matches_reference_surface():
    assert r2splat_b200.__all__ == ["__version__", "rasterize_fwd", "rasterize_bwd", "voxelize_fwd",
                                    "voxelize_bwd", "ParameterGradients"]
    assert not hasattr(r2splat_b200, "rasterize")
    import r2splat_b200.cuda as cuda

    assert LOW_LEVEL <= set(cuda.__all__)
    for name in LOW_LEVEL:
        assert callable(getattr(cuda, name))


def test_library_loads_and_exports_every_header_symbol():
    functions = header_functions()
    assert len(functions) >= 40
    lib = _backend.library()
    assert lib.r2s_abi_version() == 1
    raw = ctypes.CDLL(str(_backend.library_path()))
    for name in functions:
        assert hasattr(raw, name), name


def test_ctypes_signatures_match_header_arity():
    functions = header_functions()
    assert set(functions) == set(_backend.SIGNATURES)
    for name, count in functions.items():
        assert len(_backend.SIGNATURES[name][1]) == count, name


def test_workspace_queries_run_without_a_gpu():
    lib = _backend.library()
    assert lib.r2s_isect_count_workspace(10_000_000) > 0
    assert lib.r2s_isect_emit_workspace(40_000_000, 65536) >= 40_000_000 * 16
    assert lib.r2s_raster_workspace(0, 64, 200_000, 1) >= 2 * 64 * 200_000 * 32
    assert lib.r2s_voxel_workspace(1, 1000, 1) >= 2 * 1000 * 128
    assert lib.r2s_voxel_pack_workspace(200_000) >= 200_000 * 16  # one 16-byte slot-table entry per primitive


@pytest.mark.parametrize("shape", [(0, 3), (True, 3), (2.5, 3), (3,), (2**30, 4)])
def test_reject_invalid_output_shape(shape):
    with pytest.raises(ValueError, match="image_size"):
        _shape("image_size", shape, 2)


@pytest.mark.parametrize("eps,radius,detach", [(-1, None, False), (math.nan, None, False), (0, 0, False),
                                               (0, math.inf, False), (0, 1, "yes")])
def test_reject_invalid_numeric_options(eps, radius, detach):
    with pytest.raises((ValueError, TypeError)):
        _options(None, eps, radius, detach)


def test_default_radius_clip_depends_on_primitive():
    assert _options(None, 1e-8, None, False) == (1e-8, 3.0)
    assert _options(torch.ones(1), 1e-8, None, False) == (1e-8, 1.0)


def test_cpu_inputs_fail_before_native_dispatch():
    values = (torch.zeros(1, 3), torch.ones(1, 4), torch.ones(1, 3), torch.ones(1))
    with pytest.raises(ValueError, match="means must be a CUDA tensor"):
        voxelize_fwd(*values, (3, 4, 5), volume_extent=(1, 1, 1))
    with pytest.raises(ValueError, match="means must be a CUDA tensor"):
        rasterize_fwd(*values, torch.eye(4)[None], torch.eye(3)[None], (4, 4))


@pytest.mark.parametrize("dtype", [torch.float16, torch.int32])
def test_unsupported_precision_fails_before_native_dispatch(dtype):
    means = torch.zeros(1, 3, dtype=dtype)
    with pytest.raises(TypeError, match="dtype"):
        voxelize_fwd(means, None, None, None, (3, 4, 5), volume_extent=(1, 1, 1))


def test_operator_without_gpu_raises_instead_of_falling_back():
    from r2splat_b200.cuda import _wrapper

    if torch.cuda.is_available():
        pytest.skip("only meaningful without a GPU")
    with pytest.raises(RuntimeError):
        _backend.call("r2s_abi_version")
    assert not _wrapper.is_cuda_extension_available()


def test_bench_eval_counting_handles_partial_tiles():
    import bench

    offsets = torch.tensor([[[0, 3], [3, 4]]], dtype=torch.int32)
    # 2x2 tiles of 16 over a 20x24 image: tile pixels 16*16, 16*8, 4*16, 4*8.
    assert bench.count_evals_2d(offsets, 6, 20, 24, 16) == 3 * 256 + 0 * 128 + 1 * 64 + 2 * 32
    off3 = torch.tensor([[[0]], [[2]]], dtype=torch.int32)
    assert bench.count_evals_3d(off3, 5, (12, 8, 8), 8) == 2 * 512 + 3 * 256
