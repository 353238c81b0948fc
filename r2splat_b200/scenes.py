"""Seeded synthetic CT scenes (the benchmark workloads and test scenes).

Primitive distributions: means ~ U[-0.5, 0.5]^3, quats ~ N(0, 1)^4
(unnormalised; normalised on the device), scales ~ exp(N(log s0, sigma_s)) per
axis, densities = softplus(N(0, 1)); optionally beta ~ U[b0, b1] and
uncertainty ~ U[0, q1]. Draws come from a CPU ``torch.Generator`` with the
given seed, in that order, then move to the device.

Cameras: views k = 0..C-1 at angle 2 pi k / C on a circle of radius R in the
z = 0 plane, looking at the origin with world up +z; camera axes are +x right,
+y down (image rows), +z forward; viewmat = [R | -R eye; 0 0 0 1] and
K = [[f, 0, cx], [0, f, cy], [0, 0, 1]].
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import torch


@dataclass
class Scene:
    means: torch.Tensor
    quats: torch.Tensor
    scales: torch.Tensor
    densities: torch.Tensor
    viewmats: torch.Tensor
    Ks: torch.Tensor
    image_size: tuple
    volume_shape: tuple
    volume_extent: tuple = (1.0, 1.0, 1.0)
    volume_center: tuple = (0.0, 0.0, 0.0)
    beta: Optional[torch.Tensor] = None
    uncertainty: Optional[torch.Tensor] = None

    @property
    def primitives(self):
        return self.means, self.quats, self.scales, self.densities

    def to(self, device=None, dtype=None):
        def move(t):
            return None if t is None else t.to(device=device, dtype=dtype if t.is_floating_point() else None)

        return Scene(move(self.means), move(self.quats), move(self.scales), move(self.densities),
                     move(self.viewmats), move(self.Ks), self.image_size, self.volume_shape, self.volume_extent,
                     self.volume_center, move(self.beta), move(self.uncertainty))


def orbit_cameras(count: int, radius: float, focal: float, width: int, height: int, cx: Optional[float] = None,
                  cy: Optional[float] = None, dtype=torch.float32):
    """Circular trajectory of ``count`` pinhole cameras looking at the origin."""
    cx = width / 2 if cx is None else cx
    cy = height / 2 if cy is None else cy
    views, intrinsics = [], []
    up = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64)
    for k in range(count):
        theta = 2 * math.pi * k / count
        eye = torch.tensor([radius * math.cos(theta), radius * math.sin(theta), 0.0], dtype=torch.float64)
        forward = -eye / eye.norm()
        right = torch.linalg.cross(forward, up)
        right = right / right.norm()
        down = torch.linalg.cross(forward, right)
        rot = torch.stack((right, down, forward))
        view = torch.eye(4, dtype=torch.float64)
        view[:3, :3] = rot
        view[:3, 3] = -rot @ eye
        views.append(view)
        intrinsics.append(torch.tensor([[focal, 0.0, cx], [0.0, focal, cy], [0.0, 0.0, 1.0]], dtype=torch.float64))
    return torch.stack(views).to(dtype), torch.stack(intrinsics).to(dtype)


def random_primitives(n: int, seed: int, scale_mean: float, scale_sigma: float, *, beta_range=None,
                      uncertainty_max=None, dtype=torch.float32):
    gen = torch.Generator().manual_seed(seed)
    means = torch.rand((n, 3), generator=gen, dtype=torch.float64) - 0.5
    quats = torch.randn((n, 4), generator=gen, dtype=torch.float64)
    scales = torch.exp(math.log(scale_mean) + scale_sigma * torch.randn((n, 3), generator=gen, dtype=torch.float64))
    densities = torch.nn.functional.softplus(torch.randn((n,), generator=gen, dtype=torch.float64))
    beta = None
    if beta_range is not None:
        lo, hi = beta_range
        beta = lo + (hi - lo) * torch.rand((n,), generator=gen, dtype=torch.float64)
    uncertainty = None
    if uncertainty_max is not None:
        uncertainty = uncertainty_max * torch.rand((n,), generator=gen, dtype=torch.float64)
    cast = (lambda t: None if t is None else t.to(dtype))
    return cast(means), cast(quats), cast(scales), cast(densities), cast(beta), cast(uncertainty)


def small_scene(dtype=torch.float32, seed: int = 0) -> Scene:
    """N=2,000, C=4 at 0/90/180/270 degrees, R=2, 64x64 (f=100), volume 32^3 of extent 1."""
    means, quats, scales, densities, _, _ = random_primitives(2000, seed, 0.03, 0.3, dtype=dtype)
    viewmats, Ks = orbit_cameras(4, 2.0, 100.0, 64, 64, dtype=dtype)
    return Scene(means, quats, scales, densities, viewmats, Ks, (64, 64), (32, 32, 32))


def ct_scene(dtype=torch.float32, seed: int = 0) -> Scene:
    """N=200,000, scales exp(N(log 0.01, 0.4)), C=64 cone-beam views at R=3, 512x512 (f=600), volume 256^3."""
    means, quats, scales, densities, _, _ = random_primitives(200_000, seed, 0.01, 0.4, dtype=dtype)
    viewmats, Ks = orbit_cameras(64, 3.0, 600.0, 512, 512, dtype=dtype)
    return Scene(means, quats, scales, densities, viewmats, Ks, (512, 512), (256, 256, 256))


def beta_scene(n: int = 500_000, cameras: int = 128, side: int = 768, focal: float = 900.0, volume: int = 384,
               dtype=torch.float32, seed: int = 0) -> Scene:
    """Beta primitives with uncertainty: beta ~ U[0.5, 4], q ~ U[0, 0.1]; defaults are the 500k/128-view/768^2 case."""
    means, quats, scales, densities, beta, unc = random_primitives(n, seed, 0.01, 0.4, beta_range=(0.5, 4.0),
                                                                   uncertainty_max=0.1, dtype=dtype)
    viewmats, Ks = orbit_cameras(cameras, 3.0, focal, side, side, dtype=dtype)
    return Scene(means, quats, scales, densities, viewmats, Ks, (side, side), (volume, volume, volume), beta=beta,
                 uncertainty=unc)


def perturbed_means(means: torch.Tensor, sigma: float = 0.005, seed: int = 2) -> torch.Tensor:
    gen = torch.Generator().manual_seed(seed)
    noise = sigma * torch.randn(means.shape, generator=gen, dtype=torch.float64)
    return (means.detach().cpu().double() + noise).to(device=means.device, dtype=means.dtype)


__all__ = ["Scene", "beta_scene", "ct_scene", "orbit_cameras", "perturbed_means", "random_primitives",
           "small_scene"]
