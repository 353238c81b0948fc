"""Error of every output and gradient against the float64 oracle: Beta primitives with uncertainty.

The sub-problem of the 500k-primitive Beta/uncertainty configuration: 4,096
primitives with its value distributions (scales exp(N(log 0.01, 0.4)), beta ~
U[0.5, 4], q ~ U[0, 0.1]), 8 views on a radius-3 orbit, 64x64 detector (focal
scaled with the detector, 900 x 64 / 768), a 32^3 volume, v_image ~ N(0, 1),
v_variance ~ N(0, 0.1), with the variance branch attached and detached. The
fp32 CUDA path is compared with the fp64 dense oracle run on the GPU. Beta
support (d^2 < 1) lies inside the default tile rectangles (radius clip 1), so
the dense oracle and the tiled path evaluate the same samples.

The error reported is max |ours - oracle| / max |oracle| per tensor; the test
prints the table as one JSON line.
"""

import json

import pytest
import torch

import r2splat_b200 as r2s
from oracle import dense
from r2splat_b200 import scenes

pytestmark = pytest.mark.gpu
FIELDS = ("means", "quats", "scales", "densities", "beta", "uncertainty")


def _problem(device):
    means, quats, scales, densities, beta, q = scenes.random_primitives(
        4096, 0, 0.01, 0.4, beta_range=(0.5, 4.0), uncertainty_max=0.1, dtype=torch.float64)
    viewmats, Ks = scenes.orbit_cameras(8, 3.0, 900.0 * 64 / 768, 64, 64, dtype=torch.float64)
    values = dict(means=means, quats=quats, scales=scales, densities=densities, beta=beta, uncertainty=q,
                  viewmats=viewmats, Ks=Ks)
    return {k: v.to(device) for k, v in values.items()}


def _err(got, want):
    scale = want.abs().max().item()
    return (got.double() - want).abs().max().item() / (scale if scale > 0 else 1.0)


@pytest.mark.parametrize("detach", [False, True])
def test_every_output_and_gradient_against_float64_oracle(device, detach):
    base = _problem(device)
    f32 = {k: v.float() for k, v in base.items()}
    gen = torch.Generator(device=device).manual_seed(1)
    table = {}
    # Projection.
    (image, var), ctx = r2s.rasterize_fwd(*[f32[k] for k in FIELDS[:4]], f32["viewmats"], f32["Ks"], (64, 64),
                                          beta=f32["beta"], uncertainty=f32["uncertainty"],
                                          detach_variance=detach)
    leaves = {k: base[k].clone().requires_grad_(True) for k in FIELDS}
    ref_image, ref_var = dense.rasterize_dense(*[leaves[k] for k in FIELDS[:4]], base["viewmats"], base["Ks"],
                                               (64, 64), beta=leaves["beta"], uncertainty=leaves["uncertainty"],
                                               eps=1e-8, detach_variance=detach, chunk=512)
    v_image = torch.randn(ref_image.shape, device=device, dtype=torch.float64, generator=gen)
    v_var = 0.1 * torch.randn(ref_var.shape, device=device, dtype=torch.float64, generator=gen)
    table["image"] = _err(image, ref_image)
    table["image_variance"] = _err(var, ref_var)
    want = torch.autograd.grad((ref_image * v_image).sum() + (ref_var * v_var).sum(), [leaves[k] for k in FIELDS])
    got = r2s.rasterize_bwd(ctx, v_image.float(), v_var.float())
    for name, w in zip(FIELDS, want):
        table[f"raster d{name}"] = _err(getattr(got, name), w)
    # Voxelization.
    (volume, vvar), vctx = r2s.voxelize_fwd(*[f32[k] for k in FIELDS[:4]], (32, 32, 32),
                                            volume_extent=(1.0, 1.0, 1.0), beta=f32["beta"],
                                            uncertainty=f32["uncertainty"], detach_variance=detach)
    leaves = {k: base[k].clone().requires_grad_(True) for k in FIELDS}
    ref_volume, ref_vvar = dense.voxelize_dense(*[leaves[k] for k in FIELDS[:4]], (32, 32, 32),
                                                volume_extent=(1.0, 1.0, 1.0), beta=leaves["beta"],
                                                uncertainty=leaves["uncertainty"], eps=1e-8,
                                                detach_variance=detach, chunk=512)
    v_volume = torch.randn(ref_volume.shape, device=device, dtype=torch.float64, generator=gen)
    v_vvar = 0.1 * torch.randn(ref_vvar.shape, device=device, dtype=torch.float64, generator=gen)
    table["volume"] = _err(volume, ref_volume)
    table["volume_variance"] = _err(vvar, ref_vvar)
    want = torch.autograd.grad((ref_volume * v_volume).sum() + (ref_vvar * v_vvar).sum(),
                               [leaves[k] for k in FIELDS])
    got = r2s.voxelize_bwd(vctx, v_volume.float(), v_vvar.float())
    for name, w in zip(FIELDS, want):
        table[f"voxel d{name}"] = _err(getattr(got, name), w)
    print(json.dumps({"detach_variance": detach, "max_error_relative_to_max": table}))
    for name, value in table.items():
        assert value < 3e-4, (name, value)  # the fp32-vs-fp64 gradient bound of the parity tests
