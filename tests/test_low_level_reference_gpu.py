"""Every low-level name of the reference's ``r2splat.cuda`` surface against the reference build.

The 40 names of the reference's ``r2splat/cuda/_wrapper.py:123-165`` (pybind
module ``ext.cpp:8-183``) are called on the same inputs through this package
(``r2splat_b200.cuda``) and through the reference's own kernels
(``oracle/_ref``). Integer outputs (tile counts, keys, ids, offsets) and the
forward images, volumes and maps must be equal bit for bit; VJPs go through the
gradient parity check (the 1e-5 / 1e-6 contract, with the float64 VJP of the
reference's own kernels deciding elements outside it). Inputs are the small
configuration (N=2,000, 4 views at 64^2, volume 32^3) and the Beta-with-
uncertainty sub-problem (4,096 primitives, 8 views at 64^2, volume 32^3).
"""

import pytest
import torch

from _parity import as_float64, assert_gradient_parity
from oracle import dense, ref_ops
from r2splat_b200 import cuda as low
from r2splat_b200 import scenes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_ops.available(), reason="reference build (oracle/_ref) not present")]

REFERENCE_NAMES = (
    "image_loss_fwd", "image_loss_bwd", "image_loss_l1_fwd", "image_loss_l1_bwd", "volume_loss_fwd",
    "volume_loss_bwd", "isect_tiles", "isect_offset_encode", "isect_tiles_3d", "isect_offset_encode_3d",
    "voxelize_to_voxels_fwd", "voxelize_to_voxels_mean_var_fwd", "voxelize_to_voxels_bwd",
    "voxelize_to_voxels_bwd_per_gaussian", "voxelize_to_voxels_mean_var_bwd_per_gaussian",
    "beta_voxelize_to_voxels_fwd", "beta_voxelize_to_voxels_mean_var_fwd", "beta_voxelize_to_voxels_bwd",
    "beta_voxelize_to_voxels_bwd_per_gaussian", "beta_voxelize_to_voxels_mean_var_bwd_per_gaussian",
    "rasterize_to_pixels_fwd", "rasterize_to_pixels_mean_var_fwd", "rasterize_to_pixels_uncertainty_bwd",
    "rasterize_to_pixels_bwd", "rasterize_to_pixels_bwd_per_gaussian", "rasterize_to_pixels_mean_var_bwd_per_gaussian",
    "beta_rasterize_to_pixels_fwd", "beta_rasterize_to_pixels_mean_var_fwd", "beta_rasterize_to_pixels_uncertainty_bwd",
    "beta_rasterize_to_pixels_bwd", "beta_rasterize_to_pixels_bwd_per_gaussian",
    "beta_rasterize_to_pixels_mean_var_bwd_per_gaussian", "conics_mu_fwd", "conics_mu_bwd",
    "world_to_image_projection_fwd", "world_to_image_projection_bwd", "parameter_transform_fwd",
    "parameter_transform_bwd", "world_to_volume_mapping_fwd", "world_to_volume_mapping_bwd",
)
CALLED: set = set()


class _Both:
    """Calls a low-level name on both builds; float64 reruns on the reference give the VJP truth."""

    def __init__(self):
        self.ref = ref_ops.load()

    def __call__(self, name, *args):
        CALLED.add(name)
        return getattr(low, name)(*args), getattr(self.ref, name)(*args)

    def truth(self, name, *args):
        return getattr(self.ref, name)(*as_float64(args))


def _tuple(x):
    return x if isinstance(x, (tuple, list)) else (x,)


def _equal(name, ours, ref):
    for i, (a, b) in enumerate(zip(_tuple(ours), _tuple(ref))):
        if a is None or b is None or (isinstance(b, torch.Tensor) and b.numel() == 0 and a is None):
            continue
        assert torch.equal(a, b), f"{name}[{i}]"


def _vjp(name, ours, ref, truth, skip_first=False):
    pairs = list(zip(_tuple(ours), _tuple(ref), _tuple(truth)))
    if skip_first:
        pairs = pairs[1:]
    for i, (a, b, t) in enumerate(pairs):
        if b is None or (isinstance(b, torch.Tensor) and b.numel() == 0):
            assert a is None or a.numel() == 0, f"{name}[{i}]"
            continue
        assert_gradient_parity(f"{name}[{i}]", a, b, t)


@pytest.fixture(scope="module")
def both():
    return _Both()


def _gaussian_case(device):
    sc = scenes.small_scene().to(device)
    sc.uncertainty = (0.1 * torch.rand(2000, generator=torch.Generator().manual_seed(5))).to(device)
    return sc


def _beta_case(device):
    sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(device)
    sc.viewmats, sc.Ks = [t.to(device) for t in scenes.orbit_cameras(8, 2.0, 100.0, 64, 64)]
    return sc


def test_geometry_names(device, both):
    gen = torch.Generator().manual_seed(3)
    sc = _gaussian_case(device)
    n, c = sc.means.shape[0], sc.viewmats.shape[0]
    (covars, ms), ref_pt = both("parameter_transform_fwd", sc.quats, sc.scales)
    _equal("parameter_transform_fwd", (covars, ms), ref_pt)
    v_cov = torch.randn((n, 6), generator=gen).to(device)
    _vjp("parameter_transform_bwd", *both("parameter_transform_bwd", sc.quats, sc.scales, v_cov),
         both.truth("parameter_transform_bwd", sc.quats, sc.scales, v_cov))
    proj, ref_proj = both("world_to_image_projection_fwd", sc.means, covars, sc.viewmats, sc.Ks, 64, 64, 1e-8, 3.0)
    _equal("world_to_image_projection_fwd", proj, ref_proj)
    m2, cov2d, radii = proj
    v_m2 = torch.randn((c, n, 2), generator=gen).to(device)
    v_c2 = torch.randn(cov2d.shape, generator=gen).to(device)
    args = (sc.means, covars, sc.viewmats, sc.Ks, 64, 64, v_m2, v_c2)
    _vjp("world_to_image_projection_bwd", *both("world_to_image_projection_bwd", *args),
         both.truth("world_to_image_projection_bwd", *args))
    cm, ref_cm = both("conics_mu_fwd", cov2d, 1e-8)
    _equal("conics_mu_fwd", cm, ref_cm)
    conics, mus = cm
    v_con = torch.randn(conics.shape, generator=gen).to(device)
    v_mu = torch.randn(mus.shape, generator=gen).to(device)
    args = (cov2d, 1e-8, conics, mus, v_con, v_mu)
    _vjp("conics_mu_bwd", *both("conics_mu_bwd", *args), both.truth("conics_mu_bwd", *args))
    ext, ctr = sc.means.new_tensor([1.0, 1.1, 0.9]), sc.means.new_tensor([0.01, -0.02, 0.03])
    vm, ref_vm = both("world_to_volume_mapping_fwd", sc.means, covars, ms, ext, ctr, 32, 30, 28, 1e-8, 3.0)
    _equal("world_to_volume_mapping_fwd", vm, ref_vm)
    v_m3 = torch.randn((n, 3), generator=gen).to(device)
    v_c3 = torch.randn((n, 6), generator=gen).to(device)
    args = (sc.means, covars, ext, ctr, 32, 30, 28, 1e-8, v_m3, v_c3)
    _vjp("world_to_volume_mapping_bwd", *both("world_to_volume_mapping_bwd", *args),
         both.truth("world_to_volume_mapping_bwd", *args))
    # Tile lists of both projections, 2D with per-axis and square radii, and 3D.
    isect, ref_isect = both("isect_tiles", m2, radii, 16, 4, 4)
    _equal("isect_tiles", isect, ref_isect)
    _equal("isect_tiles square radii", *both("isect_tiles", m2, radii[..., 1].contiguous(), 16, 4, 4))
    _equal("isect_offset_encode", *both("isect_offset_encode", isect[1], c, 4, 4))
    isect3, ref_isect3 = both("isect_tiles_3d", vm[0], vm[2], 8, 4, 4, 4)
    _equal("isect_tiles_3d", isect3, ref_isect3)
    _equal("isect_offset_encode_3d", *both("isect_offset_encode_3d", isect3[1], 4, 4, 4))


def _raster_operands(both, sc):
    ref = both.ref
    covars, _ = ref.parameter_transform_fwd(sc.quats, sc.scales)
    w, h = sc.image_size[1], sc.image_size[0]
    c = sc.viewmats.shape[0]
    m2, cov2d, radii = ref.world_to_image_projection_fwd(sc.means, covars, sc.viewmats, sc.Ks, w, h, 1e-8,
                                                         3.0 if sc.beta is None else 1.0)
    conics, mus = ref.conics_mu_fwd(cov2d, 1e-8)
    opac = sc.densities.unsqueeze(0).expand(c, -1).contiguous()
    _, ids, fids = ref.isect_tiles(m2, radii, 16, (w + 15) // 16, (h + 15) // 16)
    offsets = ref.isect_offset_encode(ids, c, (w + 15) // 16, (h + 15) // 16)
    betas = None if sc.beta is None else (sc.beta + 0.5).unsqueeze(0).expand(c, -1).contiguous()
    return m2, conics, opac, mus, betas, offsets, ids, fids, w, h


@pytest.mark.parametrize("kind", ["gaussian", "beta"])
def test_raster_names(device, both, kind):
    sc = _gaussian_case(device) if kind == "gaussian" else _beta_case(device)
    m2, conics, opac, mus, betas, offsets, ids, fids, w, h = _raster_operands(both, sc)
    p = "" if kind == "gaussian" else "beta_"
    ops = (m2, conics, opac, mus) + (() if betas is None else (betas,))
    unc = sc.uncertainty
    _equal(p + "rasterize_to_pixels_fwd", *both(p + "rasterize_to_pixels_fwd", *ops, offsets, fids, w, h, 16))
    _equal(p + "rasterize_to_pixels_mean_var_fwd",
           *both(p + "rasterize_to_pixels_mean_var_fwd", *ops, unc, offsets, fids, w, h, 16))
    gen = torch.Generator().manual_seed(7)
    c = m2.shape[0]
    v = torch.randn((c, h, w), generator=gen).to(device)
    vv = (0.1 * torch.randn((c, h, w), generator=gen)).to(device)
    name = p + "rasterize_to_pixels_uncertainty_bwd"
    args = ops + (offsets, fids, vv, w, h, 16)
    _vjp(name, *both(name, *args), both.truth(name, *args))
    for absgrad in (False, True):
        name = p + "rasterize_to_pixels_bwd"
        args = ops + (offsets, fids, v, w, h, 16, absgrad)
        _vjp(name, *both(name, *args), both.truth(name, *args), skip_first=not absgrad)
        name = p + "rasterize_to_pixels_bwd_per_gaussian"
        args = ops + (offsets, ids, fids, v, w, h, 16, absgrad)
        _vjp(name, *both(name, *args), both.truth(name, *args), skip_first=not absgrad)
    name = p + "rasterize_to_pixels_mean_var_bwd_per_gaussian"
    for tail in ((w, h, 16, True), (unc, False, w, h, 16, False), (unc, True, w, h, 16, False)):
        args = ops + (offsets, ids, fids, v, vv) + tail
        ours, ref = both(name, *args)
        _vjp(name, ours, ref, both.truth(name, *args), skip_first=tail[-1] is False)


@pytest.mark.parametrize("kind", ["gaussian", "beta"])
def test_absgrad_values_match_the_dense_oracle(device, both, kind):
    """absgrad (the first slot with absgrad=True) against the float64 dense statistic with the same tile lists."""
    sc = _gaussian_case(device) if kind == "gaussian" else _beta_case(device)
    m2, conics, opac, mus, betas, offsets, ids, fids, w, h = _raster_operands(both, sc)
    p = "" if kind == "gaussian" else "beta_"
    ops = (m2, conics, opac, mus) + (() if betas is None else (betas,))
    v = torch.randn((m2.shape[0], h, w), generator=torch.Generator().manual_seed(8)).to(device)
    mask = dense.tile_mask_2d(fids.cpu(), offsets.cpu(), m2.shape[1], m2.shape[0], h, w, 16)
    want = dense.absgrad_dense(m2.double().cpu(), conics.double().cpu(), opac.double().cpu(), mus.double().cpu(),
                               v.double().cpu(), betas=None if betas is None else betas.double().cpu(),
                               tile_mask=mask)
    pixel = getattr(low, p + "rasterize_to_pixels_bwd")(*ops, offsets, fids, v, w, h, 16, True)[0]
    primitive = getattr(low, p + "rasterize_to_pixels_bwd_per_gaussian")(*ops, offsets, ids, fids, v, w, h, 16,
                                                                        True)[0]
    assert float(want.abs().max()) > 0
    for got in (pixel, primitive):
        torch.testing.assert_close(got.double().cpu(), want, rtol=2e-5, atol=2e-5 * float(want.abs().max()))


def _voxel_operands(both, sc):
    ref = both.ref
    covars, ms = ref.parameter_transform_fwd(sc.quats, sc.scales)
    d, h, w = sc.volume_shape
    ext, ctr = sc.means.new_ones(3), sc.means.new_zeros(3)
    m3, conics, radii = ref.world_to_volume_mapping_fwd(sc.means, covars, ms, ext, ctr, w, h, d, 1e-8,
                                                        3.0 if sc.beta is None else 1.0)
    t = (w + 7) // 8, (h + 7) // 8, (d + 7) // 8
    _, ids, fids = ref.isect_tiles_3d(m3, radii, 8, *t)
    offsets = ref.isect_offset_encode_3d(ids, *t)
    return m3, conics, ids, fids, offsets, w, h, d


@pytest.mark.parametrize("kind", ["gaussian", "beta"])
def test_voxel_names(device, both, kind):
    sc = _gaussian_case(device) if kind == "gaussian" else _beta_case(device)
    m3, conics, ids, fids, offsets, w, h, d = _voxel_operands(both, sc)
    p = "" if kind == "gaussian" else "beta_"
    ops = (m3, conics, sc.densities) + (() if sc.beta is None else (sc.beta,))
    unc = sc.uncertainty
    _equal(p + "voxelize_to_voxels_fwd", *both(p + "voxelize_to_voxels_fwd", *ops, offsets, fids, w, h, d, 8))
    _equal(p + "voxelize_to_voxels_mean_var_fwd",
           *both(p + "voxelize_to_voxels_mean_var_fwd", *ops, unc, offsets, fids, w, h, d, 8))
    gen = torch.Generator().manual_seed(9)
    v = torch.randn((d, h, w), generator=gen).to(device)
    vv = (0.1 * torch.randn((d, h, w), generator=gen)).to(device)
    name = p + "voxelize_to_voxels_bwd"
    args = ops + (offsets, fids, v, w, h, d, 8)
    _vjp(name, *both(name, *args), both.truth(name, *args))
    name = p + "voxelize_to_voxels_bwd_per_gaussian"
    args = ops + (offsets, ids, fids, v, w, h, d, 8)
    _vjp(name, *both(name, *args), both.truth(name, *args))
    name = p + "voxelize_to_voxels_mean_var_bwd_per_gaussian"
    for tail in ((w, h, d, 8), (unc, False, w, h, d, 8), (unc, True, w, h, d, 8)):
        args = ops + (offsets, ids, fids, v, vv) + tail
        _vjp(name, *both(name, *args), both.truth(name, *args))


def test_loss_names(device, both):
    gen = torch.Generator().manual_seed(10)
    pred = torch.randn(3, 17, 19, generator=gen).to(device)
    target = torch.randn(3, 17, 19, generator=gen).to(device)
    g = torch.full((1,), 0.7, device=device)
    for fwd, bwd in (("image_loss_fwd", "image_loss_bwd"), ("image_loss_l1_fwd", "image_loss_l1_bwd")):
        ours, ref = both(fwd, pred, target, 2.0)
        assert torch.equal(ours[2], ref[2]), fwd  # the per-pixel map
        for a, b in zip(ours[:2], ref[:2]):
            torch.testing.assert_close(a, b, rtol=1e-6, atol=1e-7)
        _equal(bwd, *both(bwd, pred, target, g, 2.0))
    vol = torch.randn(2, 11, 13, 17, generator=gen).to(device)
    ours, ref = both("volume_loss_fwd", vol, 0.05)
    assert torch.equal(ours[2], ref[2])
    for a, b in zip(ours[:2], ref[:2]):
        torch.testing.assert_close(a, b, rtol=1e-6, atol=1e-7)
    _equal("volume_loss_bwd", *both("volume_loss_bwd", vol, g, 0.05))
    assert low.is_cuda_extension_available() and both.ref is not None
    CALLED.add("is_cuda_extension_available")


def test_zz_every_reference_name_was_called():
    """Runs last in this module: each of the reference's 40 low-level names went through a comparison."""
    missing = sorted(set(REFERENCE_NAMES) - CALLED)
    assert not missing, missing
    assert len(REFERENCE_NAMES) == 40
