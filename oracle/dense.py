"""Dense float64 oracle for projection and voxelization -- TEST INFRASTRUCTURE ONLY.

Restates the reference's independent test oracle (``tests/_reference.py``):
``covariance_matrix`` :13-21, the profiles and thresholds :24-42,
``voxelize_reference`` :45-67 and ``rasterize_reference`` :70-116. Every
(primitive, sample) pair is evaluated; there is no tile selection, so results
match the CUDA path exactly only when every contributing sample lies inside the
primitive's tile rectangle (use a large ``radius_clip`` on the CUDA side, or
pass ``tile_mask`` built from the CUDA intersection lists).

All functions are differentiable with torch autograd; run them in float64 on
the CPU. ``chunk`` bounds memory by summing over primitive chunks (the sums
are linear in the primitives).
"""

from __future__ import annotations

import math
from typing import Optional

import torch


def rotation_matrix(quats: torch.Tensor) -> torch.Tensor:
    """Rotation matrices [N,3,3] of wxyz quaternions (normalised first)."""
    q = quats / torch.linalg.vector_norm(quats, dim=-1, keepdim=True)
    w, x, y, z = q.unbind(-1)
    rows = [
        1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
        2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
        2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y),
    ]
    return torch.stack(rows, dim=-1).reshape(*q.shape[:-1], 3, 3)


def covariance_matrix(quats: torch.Tensor, scales: torch.Tensor) -> torch.Tensor:
    """R diag(s^2) R^T for each primitive (``_reference.py:13-21``)."""
    rot = rotation_matrix(quats)
    return rot @ torch.diag_embed(scales.square()) @ rot.transpose(-1, -2)


def _profile(distance, exponent):
    """exp(-d/2) (Gaussian) or (1 - d)^exponent on [0, 1) (Beta) (``_reference.py:24-30``)."""
    if exponent is None:
        return torch.exp(-0.5 * distance)
    inside = (distance >= 0) & (distance < 1)
    base = torch.where(inside, 1 - distance, torch.ones_like(distance))
    return torch.where(inside, base.pow(exponent), torch.zeros_like(distance))


def _threshold(contribution, threshold):
    return torch.where(contribution.abs() >= threshold, contribution, torch.zeros_like(contribution))


def voxelize_dense(means, quats, scales, densities, volume_shape, *, volume_extent, volume_center=(0, 0, 0),
                   beta=None, uncertainty=None, eps=0.0, detach_variance=False, chunk: int = 4096):
    """Density sampled at voxel centres; ``eps`` is in voxel units squared (``_reference.py:45-67``).

    Returns the volume, or (volume, variance) with uncertainty.
    """
    depth, height, width = volume_shape
    extent = torch.as_tensor(volume_extent, device=means.device, dtype=means.dtype)
    center = torch.as_tensor(volume_center, device=means.device, dtype=means.dtype)
    dims = means.new_tensor([width, height, depth])
    voxel = extent / dims
    axes = [center[a] + ((torch.arange(s, device=means.device, dtype=means.dtype) + 0.5) / s - 0.5) * extent[a]
            for a, s in enumerate((width, height, depth))]
    zz, yy, xx = torch.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    grid = torch.stack((xx, yy, zz), dim=-1)
    threshold = 1e-6 if beta is None else 1e-5
    mean_total = means.new_zeros(tuple(volume_shape))
    var_total = means.new_zeros(tuple(volume_shape)) if uncertainty is not None else None
    for lo in range(0, means.shape[0], chunk):
        hi = min(lo + chunk, means.shape[0])
        cov = covariance_matrix(quats[lo:hi], scales[lo:hi]) + torch.diag(eps * voxel.square())
        precision = torch.linalg.inv(cov)
        delta = grid[None] - means[lo:hi, None, None, None]
        distance = torch.einsum("ndhwi,nij,ndhwj->ndhw", delta, precision, delta)
        exponent = None if beta is None else beta[lo:hi, None, None, None]
        contribution = densities[lo:hi, None, None, None] * _profile(distance, exponent)
        contribution = _threshold(contribution, threshold)
        mean_total = mean_total + contribution.sum(0)
        if uncertainty is not None:
            branch = contribution.detach() if detach_variance else contribution
            var_total = var_total + (uncertainty[lo:hi, None, None, None] * branch.square()).sum(0)
    return mean_total if uncertainty is None else (mean_total, var_total)


def rasterize_dense(means, quats, scales, densities, viewmats, Ks, image_size, *, beta=None, uncertainty=None,
                    eps=0.0, detach_variance=False, chunk: int = 1024, tile_mask: Optional[torch.Tensor] = None):
    """Line integrals of the camera/ray-coordinate densities (``_reference.py:70-116``).

    ``tile_mask`` (optional, bool [C,N,H,W]) restricts each primitive to the
    pixels the CUDA intersection lists assign to it.
    """
    height, width = image_size
    rotation, translation = viewmats[:, :3, :3], viewmats[:, :3, 3]
    yy, xx = torch.meshgrid(torch.arange(height, device=means.device, dtype=means.dtype) + 0.5,
                            torch.arange(width, device=means.device, dtype=means.dtype) + 0.5, indexing="ij")
    pixels = torch.stack((xx, yy), dim=-1)
    fx, fy, cx, cy = (Ks[:, i, j, None] for i, j in ((0, 0), (1, 1), (0, 2), (1, 2)))
    cams = viewmats.shape[0]
    mean_total = means.new_zeros((cams, height, width))
    var_total = means.new_zeros((cams, height, width)) if uncertainty is not None else None
    for lo in range(0, means.shape[0], chunk):
        hi = min(lo + chunk, means.shape[0])
        m = means[lo:hi]
        camera = torch.einsum("cij,nj->cni", rotation, m) + translation[:, None]
        x, y, z = camera.unbind(dim=-1)
        visible = z > 0.01
        z = torch.where(visible, z, torch.ones_like(z))
        tx = z * torch.clamp(x / z, min=-(cx + 0.15 * width) / fx, max=(1.15 * width - cx) / fx)
        ty = z * torch.clamp(y / z, min=-(cy + 0.15 * height) / fy, max=(1.15 * height - cy) / fy)
        zero = torch.zeros_like(z)
        ray = torch.stack((tx, ty, z), dim=-1)
        jac = torch.stack((
            torch.stack((fx / z, zero, -fx * tx / z.square()), dim=-1),
            torch.stack((zero, fy / z, -fy * ty / z.square()), dim=-1),
            ray / torch.linalg.vector_norm(ray, dim=-1, keepdim=True),
        ), dim=-2)
        cov = covariance_matrix(quats[lo:hi], scales[lo:hi])
        cam_cov = rotation[:, None] @ cov[None] @ rotation[:, None].transpose(-1, -2)
        projected = jac @ cam_cov @ jac.transpose(-1, -2) + eps * torch.eye(3, device=means.device,
                                                                            dtype=means.dtype)
        footprint = projected[..., :2, :2]
        cross = projected[..., :2, 2]
        ray_var = projected[..., 2, 2] - (cross * torch.linalg.solve(footprint, cross[..., None]).squeeze(-1)).sum(-1)
        path = torch.sqrt(2 * math.pi * ray_var)
        if beta is not None:
            g = beta[lo:hi].double()
            log_integral = math.lgamma(0.5) + torch.lgamma(g + 1) - torch.lgamma(g + 1.5)
            path = path * (log_integral.exp() / math.sqrt(2 * math.pi)).to(beta.dtype)[None]
        centre = torch.stack((fx * x / z + cx, fy * y / z + cy), dim=-1)
        delta = pixels[None, None] - centre[:, :, None, None]
        distance = torch.einsum("cnhwi,cnij,cnhwj->cnhw", delta, torch.linalg.inv(footprint), delta)
        exponent = None if beta is None else (beta[lo:hi] + 0.5)[None, :, None, None]
        contribution = (densities[lo:hi][None] * path)[:, :, None, None] * _profile(distance, exponent)
        contribution = torch.where(visible[:, :, None, None], contribution, torch.zeros_like(contribution))
        if tile_mask is not None:
            contribution = torch.where(tile_mask[:, lo:hi], contribution, torch.zeros_like(contribution))
        contribution = _threshold(contribution, 1e-5)
        mean_total = mean_total + contribution.sum(1)
        if uncertainty is not None:
            branch = contribution.detach() if detach_variance else contribution
            var_total = var_total + (uncertainty[lo:hi][None, :, None, None] * branch.square()).sum(1)
    return mean_total if uncertainty is None else (mean_total, var_total)


def absgrad_dense(means2d, conics, opacities, mus, v_image, *, betas=None, tile_mask=None):
    """Per (camera, primitive) sum over pixels of |d loss / d means2d| of each pixel's term, float64.

    The densification statistic the reference's raster VJPs return in their
    first slot when ``absgrad`` is set: each pixel's mean-position adjoint is
    taken in absolute value per component before the sum
    (``RasterizeToPixelsBwd.cu:216-221`` pixel mode, ``:459-462`` per-primitive
    mode; the reference's test oracle ``tests/test_beta_low_level_numeric.py:113-149``).
    Inputs are the low-level 2D operands: ``means2d [C,N,2]``, ``conics
    [C,N,3]`` (a, b, c), ``opacities [C,N]``, ``mus [C,N]``, ``v_image [C,H,W]``,
    and for Beta primitives the exponents ``betas [C,N]``. Gaussian samples
    count when sigma >= 0 and |alpha| >= 1e-5; Beta samples when 0 <= d^2 < 1
    and |alpha| >= 1e-5. ``tile_mask`` (bool [C,N,H,W]) restricts each pair to
    the pixels of its listed tiles.
    """
    cams, height, width = v_image.shape
    yy, xx = torch.meshgrid(torch.arange(height, dtype=means2d.dtype) + 0.5,
                            torch.arange(width, dtype=means2d.dtype) + 0.5, indexing="ij")
    dx = xx[None, None] - means2d[..., 0, None, None]
    dy = yy[None, None] - means2d[..., 1, None, None]
    a, b, c = (conics[..., i, None, None] for i in range(3))
    om = (opacities * mus)[..., None, None]
    v = v_image[:, None]
    if betas is None:
        sigma = 0.5 * (a * dx * dx + c * dy * dy) + b * dx * dy
        alpha = om * torch.exp(-sigma)
        valid = (sigma >= 0) & (alpha.abs() >= 1e-5)
        v_sigma = -v * alpha
        vx = -v_sigma * (a * dx + b * dy)
        vy = -v_sigma * (c * dy + b * dx)
    else:
        ex, ey = -dx, -dy  # the Beta form measures from the pixel to the centre
        d2 = a * ex * ex + 2.0 * b * ex * ey + c * ey * ey
        h = 1.0 - d2
        inside = (d2 >= 0) & (h > 0)
        hp = h.clamp_min(0)
        beta = betas[..., None, None]
        alpha = torch.where(inside, om * hp.pow(beta), torch.zeros_like(h))
        valid = inside & (alpha.abs() >= 1e-5)
        v_d2 = -om * beta * torch.where(inside, hp.pow(beta - 1.0), torch.zeros_like(h)) * v
        vx = 2.0 * v_d2 * (a * ex + b * ey)
        vy = 2.0 * v_d2 * (b * ex + c * ey)
    if tile_mask is not None:
        valid = valid & tile_mask
    zero = torch.zeros_like(vx)
    return torch.stack((torch.where(valid, vx.abs(), zero).sum((-2, -1)),
                        torch.where(valid, vy.abs(), zero).sum((-2, -1))), dim=-1)


def tile_mask_2d(flatten_ids, offsets, n_primitives, cameras, height, width, tile_size):
    """bool [C,N,H,W]: pixel belongs to a tile that lists the (camera, primitive) pair."""
    import numpy as np

    fid = np.asarray(flatten_ids, dtype=np.int64)
    off = np.asarray(offsets, dtype=np.int64).reshape(-1)
    tiles_y, tiles_x = (height + tile_size - 1) // tile_size, (width + tile_size - 1) // tile_size
    mask = np.zeros((cameras, n_primitives, height, width), dtype=bool)
    ends = np.append(off[1:], len(fid))
    for key in range(len(off)):
        cam, tile = divmod(key, tiles_y * tiles_x)
        ty, tx = divmod(tile, tiles_x)
        for g in fid[off[key]:ends[key]]:
            n = g - cam * n_primitives
            mask[cam, n, ty * tile_size:(ty + 1) * tile_size, tx * tile_size:(tx + 1) * tile_size] = True
    return torch.from_numpy(mask)


__all__ = ["absgrad_dense", "covariance_matrix", "rasterize_dense", "rotation_matrix", "tile_mask_2d",
           "voxelize_dense"]
