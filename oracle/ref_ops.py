"""The reference's own CUDA build, loaded as a checker -- TEST INFRASTRUCTURE ONLY.

``oracle/build_ref.py`` compiles the reference's operator sources unmodified
into ``oracle/_ref/r2splat_ref_csrc*.so`` (a torch extension exposing the 40
pybind names of ``ext.cpp:8-183``). ``load()`` imports that module;
``explicit_rasterize_fwd/bwd`` and ``explicit_voxelize_fwd/bwd`` restate the
call sequence of the reference's ``explicit.py`` (:160-183, :204-241,
:286-307, :331-350) on top of it, so parity tests and the reference bench arm
run the reference kernels exactly as the reference's public API does and can
read the intermediate buffers. ``load_package()`` imports the reference's own
Python package as staged by ``oracle/build_ref.py`` (``oracle/_ref/py``) with
``r2splat.csrc`` bound to the compiled module, so the reference bench arm runs
the reference's unmodified ``explicit.py`` on the reference's kernels.
"""

from __future__ import annotations

import importlib.machinery
import importlib.util
import sys
from pathlib import Path

import torch

_REF_DIR = Path(__file__).resolve().parent / "_ref"
_module = None


def available() -> bool:
    return bool(sorted(_REF_DIR.glob("r2splat_ref_csrc*.so")))


def load():
    """Imports the compiled reference extension (raises FileNotFoundError if not built)."""
    global _module
    if _module is not None:
        return _module
    hits = sorted(_REF_DIR.glob("r2splat_ref_csrc*.so"))
    if not hits:
        raise FileNotFoundError(f"no reference build under {_REF_DIR}; run python oracle/build_ref.py")
    loader = importlib.machinery.ExtensionFileLoader("r2splat_ref_csrc", str(hits[0]))
    spec = importlib.util.spec_from_file_location("r2splat_ref_csrc", str(hits[0]), loader=loader)
    module = importlib.util.module_from_spec(spec)
    loader.exec_module(module)
    _module = module
    return module


def package_available() -> bool:
    return available() and (_REF_DIR / "py" / "r2splat" / "explicit.py").is_file()


def load_package():
    """The reference's own ``r2splat`` package with its extension bound to ``load()``'s module.

    The reference resolves its kernels with ``importlib.import_module("r2splat.csrc")``
    (``r2splat/cuda/_backend.py:29``); registering the compiled module under that
    name beforehand makes that import return it. Raises FileNotFoundError when
    either the build or the staged package is missing.
    """
    root = _REF_DIR / "py"
    if not (root / "r2splat" / "explicit.py").is_file():
        raise FileNotFoundError(f"no staged reference package under {root}; run python oracle/build_ref.py")
    module = load()
    sys.modules.setdefault("r2splat.csrc", module)
    if str(root) not in sys.path:
        sys.path.insert(0, str(root))
    import r2splat

    if not r2splat.cuda.is_cuda_extension_available():
        raise RuntimeError("the reference package did not bind its CUDA extension")
    return r2splat


def _ratio(beta):
    from r2splat_b200._beta import beta_path_ratio

    return beta_path_ratio(beta)


def _log_grad(beta):
    from r2splat_b200._beta import beta_path_log_grad

    return beta_path_log_grad(beta)


@torch.no_grad()
def explicit_rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, *, beta=None,
                           uncertainty=None, eps=1e-8, radius_clip=None):
    """Reference explicit.py:160-183 on the reference kernels. Returns (output, saved)."""
    ref = load()
    height, width = image_size
    if radius_clip is None:
        radius_clip = 3.0 if beta is None else 1.0
    cameras = viewmats.shape[0]
    covars, _ = ref.parameter_transform_fwd(quats, scales)
    mapped, cov2d, radii = ref.world_to_image_projection_fwd(means, covars, viewmats, Ks, width, height, eps,
                                                             radius_clip)
    conics, base_mus = ref.conics_mu_fwd(cov2d, eps)
    opacity = densities.unsqueeze(0).expand(cameras, -1).contiguous()
    mus, beta2d, ratio = base_mus, None, None
    if beta is not None:
        ratio = _ratio(beta)
        mus = base_mus * ratio.unsqueeze(0)
        beta2d = (beta + 0.5).unsqueeze(0).expand(cameras, -1).contiguous()
    tiles_x, tiles_y = (width + 15) // 16, (height + 15) // 16
    tiles_per_gauss, isect_ids, flatten_ids = ref.isect_tiles(mapped, radii, 16, tiles_x, tiles_y)
    offsets = ref.isect_offset_encode(isect_ids, cameras, tiles_x, tiles_y)
    prefix = "beta_" if beta is not None else ""
    args = (mapped, conics, opacity, mus) + (() if beta is None else (beta2d,))
    if uncertainty is None:
        output = getattr(ref, prefix + "rasterize_to_pixels_fwd")(*args, offsets, flatten_ids, width, height, 16)
    else:
        output = getattr(ref, prefix + "rasterize_to_pixels_mean_var_fwd")(*args, uncertainty, offsets,
                                                                          flatten_ids, width, height, 16)
    saved = dict(covars=covars, mapped=mapped, cov2d=cov2d, radii=radii, conics=conics, base_mus=base_mus, mus=mus,
                 opacity=opacity, beta2d=beta2d, ratio=ratio, offsets=offsets, isect_ids=isect_ids,
                 flatten_ids=flatten_ids, tiles_per_gauss=tiles_per_gauss, width=width, height=height, eps=eps,
                 viewmats=viewmats, Ks=Ks)
    return output, saved


@torch.no_grad()
def explicit_rasterize_bwd(saved, means, quats, scales, beta, uncertainty, v_image, v_variance=None,
                           detach_variance=False, mode="primitive"):
    """Reference explicit.py:204-241 on the reference kernels -> tuple of parameter gradients."""
    ref = load()
    b = saved
    width, height = b["width"], b["height"]
    if v_image is None:
        v_image = means.new_zeros((b["viewmats"].shape[0], height, width))
    prefix = "beta_" if beta is not None else ""
    args = (b["mapped"], b["conics"], b["opacity"], b["mus"]) + (() if beta is None else (b["beta2d"],))
    if v_variance is not None:
        grads = getattr(ref, prefix + "rasterize_to_pixels_mean_var_bwd_per_gaussian")(
            *args, b["offsets"], b["isect_ids"], b["flatten_ids"], v_image, v_variance, uncertainty,
            detach_variance, width, height, 16, False)
        v_unc = grads[-1]
    else:
        primitive = mode == "primitive"
        ids = (b["offsets"],) + ((b["isect_ids"],) if primitive else ()) + (b["flatten_ids"],)
        fn = prefix + "rasterize_to_pixels_bwd" + ("_per_gaussian" if primitive else "")
        grads = getattr(ref, fn)(*args, *ids, v_image, width, height, 16, False)
        v_unc = None if uncertainty is None else torch.zeros_like(uncertainty)
    v_mapped, v_conics, v_dens, v_mus = grads[1:5]
    v_beta = None
    if beta is not None:
        v_beta = grads[5].sum(dim=0)
        v_beta += (v_mus * b["mus"]).sum(dim=0) * _log_grad(beta)
        v_mus = (v_mus * b["ratio"].unsqueeze(0)).contiguous()
    v_cov2d = ref.conics_mu_bwd(b["cov2d"], b["eps"], b["conics"], b["base_mus"], v_conics.contiguous(),
                                v_mus.contiguous())
    v_means, v_covars = ref.world_to_image_projection_bwd(means, b["covars"], b["viewmats"], b["Ks"], width,
                                                          height, v_mapped.contiguous(), v_cov2d.contiguous())
    v_quats, v_scales = ref.parameter_transform_bwd(quats, scales, v_covars.contiguous())
    return v_means, v_quats, v_scales, v_dens.sum(dim=0), v_beta, v_unc


@torch.no_grad()
def explicit_voxelize_fwd(means, quats, scales, densities, volume_shape, *, volume_extent, volume_center=(0, 0, 0),
                          beta=None, uncertainty=None, eps=1e-8, radius_clip=None):
    """Reference explicit.py:286-307 on the reference kernels. Returns (output, saved)."""
    ref = load()
    depth, height, width = volume_shape
    if radius_clip is None:
        radius_clip = 3.0 if beta is None else 1.0
    extent = torch.as_tensor(volume_extent, device=means.device, dtype=means.dtype)
    center = torch.as_tensor(volume_center, device=means.device, dtype=means.dtype)
    covars, max_scales = ref.parameter_transform_fwd(quats, scales)
    mapped, conics, radii = ref.world_to_volume_mapping_fwd(means, covars, max_scales, extent, center, width, height,
                                                            depth, eps, radius_clip)
    tiles_x, tiles_y, tiles_z = (width + 7) // 8, (height + 7) // 8, (depth + 7) // 8
    tiles_per_gauss, isect_ids, flatten_ids = ref.isect_tiles_3d(mapped, radii, 8, tiles_x, tiles_y, tiles_z)
    offsets = ref.isect_offset_encode_3d(isect_ids, tiles_x, tiles_y, tiles_z)
    prefix = "beta_" if beta is not None else ""
    args = (mapped, conics, densities) + (() if beta is None else (beta,))
    if uncertainty is None:
        output = getattr(ref, prefix + "voxelize_to_voxels_fwd")(*args, offsets, flatten_ids, width, height, depth, 8)
    else:
        output = getattr(ref, prefix + "voxelize_to_voxels_mean_var_fwd")(*args, uncertainty, offsets, flatten_ids,
                                                                         width, height, depth, 8)
    saved = dict(covars=covars, mapped=mapped, conics=conics, radii=radii, offsets=offsets, isect_ids=isect_ids,
                 flatten_ids=flatten_ids, tiles_per_gauss=tiles_per_gauss, extent=extent, center=center,
                 shape=(depth, height, width), eps=eps)
    return output, saved


@torch.no_grad()
def explicit_voxelize_bwd(saved, means, quats, scales, densities, beta, uncertainty, v_volume, v_variance=None,
                          detach_variance=False, mode="primitive"):
    """Reference explicit.py:331-350 on the reference kernels."""
    ref = load()
    b = saved
    depth, height, width = b["shape"]
    if v_volume is None:
        v_volume = means.new_zeros(b["shape"])
    prefix = "beta_" if beta is not None else ""
    args = (b["mapped"], b["conics"], densities) + (() if beta is None else (beta,))
    if v_variance is not None:
        grads = getattr(ref, prefix + "voxelize_to_voxels_mean_var_bwd_per_gaussian")(
            *args, b["offsets"], b["isect_ids"], b["flatten_ids"], v_volume, v_variance, uncertainty,
            detach_variance, width, height, depth, 8)
        v_unc = grads[-1]
    else:
        primitive = mode == "primitive"
        ids = (b["offsets"],) + ((b["isect_ids"],) if primitive else ()) + (b["flatten_ids"],)
        fn = prefix + "voxelize_to_voxels_bwd" + ("_per_gaussian" if primitive else "")
        grads = getattr(ref, fn)(*args, *ids, v_volume, width, height, depth, 8)
        v_unc = None if uncertainty is None else torch.zeros_like(uncertainty)
    v_mapped, v_conics, v_dens = grads[:3]
    v_beta = None if beta is None else grads[3]
    v_means, v_covars = ref.world_to_volume_mapping_bwd(means, b["covars"], b["extent"], b["center"], width, height,
                                                        depth, b["eps"], v_mapped.contiguous(), v_conics.contiguous())
    v_quats, v_scales = ref.parameter_transform_bwd(quats, scales, v_covars.contiguous())
    return v_means, v_quats, v_scales, v_dens, v_beta, v_unc


__all__ = ["available", "load_package", "package_available", "explicit_rasterize_bwd", "explicit_rasterize_fwd", "explicit_voxelize_bwd",
           "explicit_voxelize_fwd", "load"]
