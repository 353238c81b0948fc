"""CUDA parity tests: the sm_100a library against the float64 oracle, the numpy
tile oracle and (when built) the reference's own CUDA kernels."""

from dataclasses import is_dataclass

import numpy as np
import pytest
import torch

import r2splat_b200 as r2s
from _parity import assert_gradient_parity as _assert_gradient_parity
from oracle import dense, losses, ref_ops, tiles
from r2splat_b200 import scenes
from r2splat_b200.cuda import _wrapper as low

pytestmark = pytest.mark.gpu
FIELDS = ("means", "quats", "scales", "densities", "beta", "uncertainty")
needs_ref = pytest.mark.skipif(not ref_ops.available(), reason="reference build (oracle/_ref) not present")


def _scene(beta, uncertainty, dtype, seed=3, n=24):
    means, quats, scales, densities, b, q = scenes.random_primitives(
        n, seed, 0.12, 0.25, beta_range=(0.8, 4.0) if beta else None, uncertainty_max=0.3 if uncertainty else None,
        dtype=torch.float64)
    viewmats, Ks = scenes.orbit_cameras(2, 2.4, 18.0, 21, 15, dtype=torch.float64)
    values = dict(means=means * 0.6, quats=quats, scales=scales, densities=densities, beta=b, uncertainty=q,
                  viewmats=viewmats, Ks=Ks)
    return values


def _to(values, device, dtype):
    return {k: None if v is None else v.to(device=device, dtype=dtype) for k, v in values.items()}


def _forward(op, values, explicit, detach=False, mode="primitive"):
    options = dict(beta=values["beta"], uncertainty=values["uncertainty"], eps=0.01, detach_variance=detach)
    prims = [values[k] for k in FIELDS[:4]]
    if explicit:
        options["backward_mode"] = mode
        options["radius_clip"] = 8.0 if values["beta"] is None else 1.0
        fn = r2s.rasterize_fwd if op == "rasterize" else r2s.voxelize_fwd
    else:
        fn = dense.rasterize_dense if op == "rasterize" else dense.voxelize_dense
    if op == "rasterize":
        return fn(*prims, values["viewmats"], values["Ks"], (15, 21), **options)
    return fn(*prims, (6, 7, 9), volume_extent=(1.6, 1.5, 1.4), volume_center=(0.02, -0.03, 0.01), **options)


def _outs(x):
    return x if isinstance(x, tuple) else (x,)


@pytest.mark.parametrize("op", ["rasterize", "voxelize"])
@pytest.mark.parametrize("beta,unc,detach,dtype,mode", [
    (False, False, False, torch.float32, "primitive"),
    (True, False, False, torch.float64, "pixel"),
    (False, False, False, torch.float64, "pixel"),
    (True, False, False, torch.float32, "primitive"),
    (False, True, False, torch.float64, "pixel"),
    (True, True, False, torch.float32, "primitive"),
    (False, True, True, torch.float32, "primitive"),
    (True, True, True, torch.float64, "pixel"),
])
def test_explicit_vjp_matches_float64_oracle(device, op, beta, unc, detach, dtype, mode):
    base = _scene(beta, unc, torch.float64)
    values = _to(base, device, dtype)
    for name in FIELDS:
        if values[name] is not None:
            values[name].requires_grad_(True)
            values[name].grad = torch.full_like(values[name], 1.25)
    out, ctx = _forward(op, values, True, detach, mode)
    leaves = {k: (v.clone().requires_grad_(True) if k in FIELDS and v is not None else v) for k, v in base.items()}
    ref = _forward(op, leaves, False, detach)
    tol = 2e-5 if dtype == torch.float32 else 2e-11
    for got, want in zip(_outs(out), _outs(ref)):
        assert got.grad_fn is None and not got.requires_grad
        torch.testing.assert_close(got.double().cpu(), want.detach(), atol=tol, rtol=tol)
    gen = torch.Generator().manual_seed(5)
    adjoints = [torch.randn(o.shape, generator=gen, dtype=torch.float64) for o in _outs(ref)]
    keys = [k for k in FIELDS if leaves.get(k) is not None]
    loss = sum((o * a).sum() for o, a in zip(_outs(ref), adjoints))
    expected = dict(zip(keys, torch.autograd.grad(loss, [leaves[k] for k in keys], allow_unused=True)))
    bwd = r2s.rasterize_bwd if op == "rasterize" else r2s.voxelize_bwd
    grads = bwd(ctx, *[a.to(device, dtype) for a in adjoints])
    assert is_dataclass(grads)
    atol, rtol = (2e-4, 3e-4) if dtype == torch.float32 else (2e-9, 2e-9)
    for name in FIELDS:
        got = getattr(grads, name)
        if name not in expected:
            assert got is None
            continue
        want = expected[name] if expected[name] is not None else torch.zeros_like(leaves[name])
        assert got.grad_fn is None and bool(torch.isfinite(got).all())
        torch.testing.assert_close(got.double().cpu(), want, atol=atol, rtol=rtol, msg=name)
    for name in FIELDS:
        if values[name] is not None:
            torch.testing.assert_close(values[name].grad, torch.full_like(values[name], 1.25))


@pytest.mark.parametrize("op", ["rasterize", "voxelize"])
def test_explicit_vjp_matches_finite_differences(device, op):
    values = _to(_scene(True, True, torch.float64), device, torch.float64)
    out, ctx = _forward(op, values, True)
    gen = torch.Generator().manual_seed(9)
    adjoints = [torch.randn(o.shape, generator=gen, dtype=torch.float64).to(device) for o in _outs(out)]
    grads = (r2s.rasterize_bwd if op == "rasterize" else r2s.voxelize_bwd)(ctx, *adjoints)
    step = 1e-5
    for name, index in {"means": (0, 0), "quats": (1, 2), "scales": (2, 1), "densities": (3,), "beta": (4,),
                        "uncertainty": (5,)}.items():
        losses_ = []
        for sign in (1, -1):
            perturbed = {k: (v.clone() if isinstance(v, torch.Tensor) else v) for k, v in values.items()}
            perturbed[name][index] += sign * step
            sampled, _ = _forward(op, perturbed, True)
            losses_.append(sum((s * a).sum() for s, a in zip(_outs(sampled), adjoints)))
        fd = (losses_[0] - losses_[1]) / (2 * step)
        analytic = getattr(grads, name)[index]
        torch.testing.assert_close(analytic, fd, atol=2e-5, rtol=2e-4, msg=name)


@pytest.mark.parametrize("op", ["rasterize", "voxelize"])
@pytest.mark.parametrize("case,detach", [("zero", False), ("mean", False), ("variance", False), ("variance", True)])
def test_optional_adjoints_and_detached_variance(device, op, case, detach):
    base = _scene(True, True, torch.float64)
    values = _to(base, device, torch.float64)
    out, ctx = _forward(op, values, True, detach)
    gen = torch.Generator().manual_seed(4)
    v_mean, v_var = [torch.randn(o.shape, generator=gen, dtype=torch.float64) for o in out]
    if case == "zero":
        v_mean = v_var = None
    elif case == "mean":
        v_var = None
    else:
        v_mean = None
    bwd = r2s.rasterize_bwd if op == "rasterize" else r2s.voxelize_bwd
    grads = bwd(ctx, None if v_mean is None else v_mean.to(device), None if v_var is None else v_var.to(device))
    if case == "zero":
        for name in FIELDS:
            assert torch.count_nonzero(getattr(grads, name)) == 0
        return
    leaves = {k: (v.clone().requires_grad_(True) if k in FIELDS and v is not None else v) for k, v in base.items()}
    ref = _forward(op, leaves, False, detach)
    weights = [torch.zeros_like(ref[0]) if v_mean is None else v_mean, torch.zeros_like(ref[1]) if v_var is None
               else v_var]
    loss = sum((o * w).sum() for o, w in zip(ref, weights))
    expected = torch.autograd.grad(loss, [leaves[k] for k in FIELDS], allow_unused=True)
    for name, want in zip(FIELDS, expected):
        want = torch.zeros_like(leaves[name]) if want is None else want
        torch.testing.assert_close(getattr(grads, name).cpu(), want, atol=2e-9, rtol=2e-9, msg=name)
    if case == "variance" and detach:
        for name in FIELDS[:-1]:
            assert torch.count_nonzero(getattr(grads, name)) == 0
        assert bool((grads.uncertainty != 0).any())


@pytest.mark.parametrize("op", ["rasterize", "voxelize"])
def test_empty_primitives_and_context_contracts(device, op):
    values = _to(_scene(True, True, torch.float64), device, torch.float64)
    empty = dict(values)
    for k in FIELDS:
        empty[k] = values[k][:0]
    out, ctx = _forward(op, empty, True)
    for o in _outs(out):
        assert torch.count_nonzero(o) == 0
    grads = (r2s.rasterize_bwd if op == "rasterize" else r2s.voxelize_bwd)(ctx, *[torch.ones_like(o) for o in _outs(out)])
    assert grads.means.shape == (0, 3)
    out, ctx = _forward(op, values, True)
    bwd = r2s.rasterize_bwd if op == "rasterize" else r2s.voxelize_bwd
    adj = [torch.ones_like(o) for o in _outs(out)]
    with pytest.raises(ValueError):
        bwd(ctx, adj[0].reshape(-1), adj[1])
    bwd(ctx, *adj)
    with pytest.raises(RuntimeError):
        bwd(ctx, *adj)
    out, ctx = _forward(op, values, True)
    values["means"].add_(0.01)
    with pytest.raises(RuntimeError):
        bwd(ctx, *[torch.ones_like(o) for o in _outs(out)])


@pytest.mark.parametrize("tile", [16, 8, 4])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_tile_lists_match_numpy_oracle_bit_exact(device, tile, dtype):
    sc = scenes.small_scene(dtype=dtype).to(device)
    covars, _ = low.parameter_transform_fwd(sc.quats, sc.scales)
    m2, _, radii = low.world_to_image_projection_fwd(sc.means, covars, sc.viewmats, sc.Ks, 64, 64, 1e-8, 3.0)
    tx = ty = 64 // tile
    counts, ids, fids = low.isect_tiles(m2, radii, tile, tx, ty)
    offsets = low.isect_offset_encode(ids, 4, tx, ty)
    c2, i2, f2 = tiles.isect_tiles_2d(m2.cpu().numpy(), radii.cpu().numpy(), tile, tx, ty)
    assert np.array_equal(counts.cpu().numpy(), c2)
    assert np.array_equal(ids.cpu().numpy(), i2)
    assert np.array_equal(fids.cpu().numpy(), f2)
    assert np.array_equal(offsets.cpu().numpy().reshape(-1), tiles.offset_encode(i2, 4 * tx * ty))
    # square radii form and 3D tiles
    counts_sq, ids_sq, fids_sq = low.isect_tiles(m2, radii[..., 0].contiguous(), tile, tx, ty)
    c3, i3, f3 = tiles.isect_tiles_2d(m2.cpu().numpy(), radii[..., 0].cpu().numpy(), tile, tx, ty)
    assert np.array_equal(ids_sq.cpu().numpy(), i3) and np.array_equal(fids_sq.cpu().numpy(), f3)
    mv, _, r3 = low.world_to_volume_mapping_fwd(sc.means, covars, covars[:, 0].contiguous(), sc.means.new_ones(3),
                                                sc.means.new_zeros(3), 32, 32, 32, 1e-8, 3.0)
    t3 = 32 // (tile // 2)
    counts, ids, fids = low.isect_tiles_3d(mv, r3, tile // 2, t3, t3, t3)
    c3, i3, f3 = tiles.isect_tiles_3d(mv.cpu().numpy(), r3.cpu().numpy(), tile // 2, t3, t3, t3)
    assert np.array_equal(counts.cpu().numpy(), c3) and np.array_equal(ids.cpu().numpy(), i3)
    assert np.array_equal(fids.cpu().numpy(), f3)
    assert np.array_equal(low.isect_offset_encode_3d(ids, t3, t3, t3).cpu().numpy().reshape(-1),
                          tiles.offset_encode(i3, t3 ** 3))


@pytest.mark.parametrize("tiles_xy", [(40, 52), (48, 48), (64, 64), (100, 100)])
def test_tile_lists_with_many_tiles_per_camera_bit_exact(device, tiles_xy):
    """More than 1024 tiles per camera (1-pixel tiles): the camera-segmented sort takes
    the tile index in two or three passes of a few bits each."""
    sc = scenes.small_scene().to(device)
    covars, _ = low.parameter_transform_fwd(sc.quats, sc.scales)
    m2, _, radii = low.world_to_image_projection_fwd(sc.means, covars, sc.viewmats, sc.Ks, 64, 64, 1e-8, 3.0)
    tx, ty = tiles_xy
    counts, ids, fids = low.isect_tiles(m2, radii, 1, tx, ty)
    c2, i2, f2 = tiles.isect_tiles_2d(m2.cpu().numpy(), radii.cpu().numpy(), 1, tx, ty)
    assert ids.numel() > 100_000
    assert np.array_equal(counts.cpu().numpy(), c2)
    assert np.array_equal(ids.cpu().numpy(), i2)
    assert np.array_equal(fids.cpu().numpy(), f2)
    offsets = low.isect_offset_encode(ids, 4, tx, ty)
    assert np.array_equal(offsets.cpu().numpy().reshape(-1), tiles.offset_encode(i2, 4 * tx * ty))


def test_3d_tile_bound_golden_cases(device):
    import json

    from conftest import GOLDEN

    spec = json.loads((GOLDEN / "tile_bounds_3d.json").read_text())
    for dtype in (torch.float32, torch.float64):
        for case in spec["cases"]:
            means = torch.tensor([case["mean"]], dtype=dtype, device=device)
            radii = torch.full((1, 3), case["radius"], dtype=torch.int32, device=device)
            counts, ids, fids = low.isect_tiles_3d(means, radii, 4, 3, 2, 4)
            assert counts.tolist() == [len(case["expected_ids"])], case["id"]
            assert ids.tolist() == case["expected_ids"], case["id"]
            assert fids.tolist() == [0] * len(case["expected_ids"])
            offsets = low.isect_offset_encode_3d(ids, 3, 2, 4)
            expected = np.searchsorted(np.asarray(case["expected_ids"], dtype=np.int64), np.arange(24))
            assert offsets.cpu().numpy().reshape(-1).tolist() == expected.tolist()


def _odd_tile_case(ndim, primitive, dtype, device):
    """Two primitives in one odd-sized tile (15 pixels / 3 voxels), dense references."""
    gen = torch.Generator().manual_seed(13 + ndim)
    size = 15 if ndim == 2 else 3
    if ndim == 2:
        means = torch.tensor([[[7.2, 7.6], [8.1, 6.8]]], dtype=torch.float64)
        conics = torch.tensor([[[0.006, 0.0002, 0.007], [0.008, -0.0003, 0.005]]], dtype=torch.float64)
        opac = torch.tensor([[1.2, 0.8]], dtype=torch.float64)
        values = [means, conics, opac, torch.tensor([[0.9, 1.1]], dtype=torch.float64)]
        if primitive == "beta":
            values.append(torch.tensor([[2.8, 3.6]], dtype=torch.float64))
    else:
        means = torch.tensor([[1.2, 1.6, 1.4], [1.7, 1.1, 1.8]], dtype=torch.float64)
        conics = torch.tensor([[0.12, 0.005, -0.002, 0.15, 0.003, 0.1], [0.1, -0.004, 0.002, 0.13, 0.005, 0.14]],
                              dtype=torch.float64)
        values = [means, conics, torch.tensor([1.2, 0.8], dtype=torch.float64)]
        if primitive == "beta":
            values.append(torch.tensor([2.3, 3.1], dtype=torch.float64))
    values = [v.requires_grad_(True) for v in values]
    unc = torch.tensor([0.2, 0.3], dtype=torch.float64, requires_grad=True)
    axis = torch.arange(size, dtype=torch.float64) + 0.5
    grid = torch.stack(torch.meshgrid(*([axis] * ndim), indexing="ij")[::-1], dim=-1)
    delta = grid.unsqueeze(0) - values[0].reshape(2, *([1] * ndim), ndim)
    idx = [[0, 1], [1, 2]] if ndim == 2 else [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
    prec = values[1].reshape(2, -1)[:, idx]
    dist = torch.einsum("n...i,nij,n...j->n...", delta, prec, delta)
    shape = (2, *([1] * ndim))
    mag = values[2].reshape(shape)
    if ndim == 2:
        mag = mag * values[3].reshape(shape)
    if primitive == "beta":
        contrib = mag * (1 - dist).clamp_min(0).pow(values[-1].reshape(shape))
    else:
        contrib = mag * torch.exp(-0.5 * dist)
    thr = 1e-6 if ndim == 3 and primitive == "gaussian" else 1e-5
    contrib = torch.where(contrib.abs() >= thr, contrib, torch.zeros_like(contrib))
    mean = contrib.sum(0)
    var = (unc.reshape(shape) * contrib.square()).sum(0)
    if ndim == 2:
        mean, var = mean.unsqueeze(0), var.unsqueeze(0)
    dev_values = [v.detach().to(device, dtype) for v in values]
    return size, values, unc, mean, var, dev_values, unc.detach().to(device, dtype)


@pytest.mark.parametrize("ndim", [2, 3])
@pytest.mark.parametrize("primitive", ["gaussian", "beta"])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_odd_tiles_forward_and_all_backward_forms(device, ndim, primitive, dtype):
    size, values, unc, ref_mean, ref_var, dv, du = _odd_tile_case(ndim, primitive, dtype, device)
    offsets = torch.zeros((1, 1, 1), dtype=torch.int32, device=device)
    fids = torch.arange(2, dtype=torch.int32, device=device)
    iids = torch.zeros(2, dtype=torch.int64, device=device)
    dims = [size] * ndim + [size]
    bwd_opts = dims + ([False] if ndim == 2 else [])
    stem = ("beta_" if primitive == "beta" else "") + ("rasterize_to_pixels" if ndim == 2 else "voxelize_to_voxels")
    call = lambda suffix, *a: getattr(low, stem + suffix)(*a)
    tol = 5e-5 if dtype == torch.float32 else 1e-10
    close = lambda a, b: torch.testing.assert_close(a.double().cpu(), b.detach(), atol=tol, rtol=tol)
    close(call("_fwd", *dv, offsets, fids, *dims), ref_mean)
    m, v = call("_mean_var_fwd", *dv, du, offsets, fids, *dims)
    close(m, ref_mean)
    close(v, ref_var)
    w = torch.linspace(0.2, 1.3, ref_mean.numel(), dtype=torch.float64).reshape(ref_mean.shape)
    wv = w.flip(-1).contiguous()
    expected = torch.autograd.grad((ref_mean * w).sum(), values, retain_graph=True)
    for grads in (call("_bwd", *dv, offsets, fids, w.to(device, dtype), *bwd_opts),
                  call("_bwd_per_gaussian", *dv, offsets, iids, fids, w.to(device, dtype), *bwd_opts)):
        grads = grads[1:] if ndim == 2 else grads
        assert len(grads) == len(expected)
        for a, b in zip(grads, expected):
            close(a, b)
    joint = torch.autograd.grad((ref_mean * w + ref_var * wv).sum(), values + [unc])
    fused = call("_mean_var_bwd_per_gaussian", *dv, offsets, iids, fids, w.to(device, dtype),
                 wv.to(device, dtype), du, False, *bwd_opts)
    fused = fused[1:] if ndim == 2 else fused
    assert len(fused) == len(joint)
    for a, b in zip(fused, joint):
        close(a, b)
    if ndim == 2:
        close(call("_uncertainty_bwd", *dv, offsets, fids, wv.to(device, dtype), *dims), joint[-1])
        plain = [x.detach() for x in values]
        want = dense.absgrad_dense(plain[0], plain[1], plain[2], plain[3], w,
                                   betas=plain[4] if primitive == "beta" else None)
        assert float(want.abs().max()) > 0
        for absgrad in (call("_bwd", *dv, offsets, fids, w.to(device, dtype), *dims[:3], True)[0],
                        call("_bwd_per_gaussian", *dv, offsets, iids, fids, w.to(device, dtype), *dims[:3], True)[0]):
            close(absgrad, want)


def test_tv_and_l1_match_oracle(device):
    case = torch.load(__import__("conftest").GOLDEN / "tv_reference.pt", weights_only=False)
    vol = case["volume"].to(device, torch.float32)
    loss, tv, tv_map = low.volume_loss_fwd(vol, 0.05)
    torch.testing.assert_close(tv.double().cpu(), case["tv"], atol=1e-6, rtol=1e-6)
    torch.testing.assert_close(loss.double().cpu(), case["loss"], atol=1e-6, rtol=1e-6)
    grad = low.volume_loss_bwd(vol, torch.ones(1, device=device), 0.05)
    torch.testing.assert_close(grad.double().cpu(), case["grad"], atol=1e-6, rtol=1e-5)
    big = torch.randn(2, 33, 40, 47, generator=torch.Generator().manual_seed(2)).to(device)
    loss, tv, tv_map = low.volume_loss_fwd(big, 0.05)
    l2, t2, m2 = losses.tv_forward(big.cpu().numpy(), 0.05)
    assert abs(float(tv) - t2) <= 1e-6 * abs(t2)
    np.testing.assert_allclose(tv_map.cpu().numpy(), m2, atol=1e-5)
    np.testing.assert_allclose(low.volume_loss_bwd(big, torch.full((1,), 0.7, device=device), 0.05).cpu().numpy(),
                               losses.tv_backward(big.cpu().numpy(), 0.7, 0.05), atol=1e-9, rtol=1e-5)
    p = torch.randn(3, 17, 19, generator=torch.Generator().manual_seed(3)).to(device)
    t = torch.randn(3, 17, 19, generator=torch.Generator().manual_seed(4)).to(device)
    loss, l1, l1_map = low.image_loss_l1_fwd(p, t, 2.0)
    lref, l1ref, mref = losses.l1_forward(p.cpu().numpy(), t.cpu().numpy(), 2.0)
    assert abs(float(l1) - l1ref) < 1e-6 and abs(float(loss) - lref) < 2e-6
    np.testing.assert_allclose(low.image_loss_l1_bwd(p, t, torch.ones(1, device=device), 2.0).cpu().numpy(),
                               losses.l1_backward(p.cpu().numpy(), t.cpu().numpy(), [1.0], 2.0), atol=1e-9)


# ----------------------------------------------------------------- reference build


def _float64(saved):
    return {k: (v.double() if isinstance(v, torch.Tensor) and v.is_floating_point() else v) for k, v in saved.items()}


def _d(t):
    return None if t is None else t.double()


def _raster_truth(saved, sc, v, vv, detach=False):
    """The float64 raster VJP of the fp32 forward in ``saved``, on the reference's float64 kernels."""
    return ref_ops.explicit_rasterize_bwd(_float64(saved), _d(sc.means), _d(sc.quats), _d(sc.scales), _d(sc.beta),
                                          _d(sc.uncertainty), _d(v), _d(vv), detach)


def _voxel_truth(saved, sc, w, wv, detach=False):
    return ref_ops.explicit_voxelize_bwd(_float64(saved), _d(sc.means), _d(sc.quats), _d(sc.scales),
                                         _d(sc.densities), _d(sc.beta), _d(sc.uncertainty), _d(w), _d(wv), detach)


@needs_ref
@pytest.mark.parametrize("beta,unc", [(False, False), (False, True), (True, False), (True, True)])
def test_explicit_matches_reference_build(device, beta, unc):
    if beta:
        sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(device)
        sc.viewmats, sc.Ks = [t.to(device) for t in scenes.orbit_cameras(8, 2.0, 100.0, 64, 64)]
        if not unc:
            sc.uncertainty = None
    else:
        sc = scenes.small_scene().to(device)
        if unc:
            sc.uncertainty = (0.1 * torch.rand(2000, generator=torch.Generator().manual_seed(5))).to(device)
    out, ctx = r2s.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                 uncertainty=sc.uncertainty)
    ref_out, saved = ref_ops.explicit_rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                                    uncertainty=sc.uncertainty)
    st = ctx.buffers["state"]
    assert torch.equal(st.isect_ids, saved["isect_ids"])
    assert torch.equal(st.flatten_ids, saved["flatten_ids"])
    assert torch.equal(st.offsets, saved["offsets"])
    for a, b in zip(_outs(out), _outs(ref_out)):
        assert torch.equal(a, b)
    gen = torch.Generator().manual_seed(11)
    v = torch.randn(_outs(out)[0].shape, generator=gen).to(device)
    vv = (0.1 * torch.randn(v.shape, generator=gen)).to(device) if unc else None
    g = r2s.rasterize_bwd(ctx, v, vv)
    r1 = ref_ops.explicit_rasterize_bwd(saved, sc.means, sc.quats, sc.scales, sc.beta, sc.uncertainty, v, vv)
    truth = _raster_truth(saved, sc, v, vv)
    for name, a, b, t in zip(FIELDS, (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty), r1, truth):
        if b is None:
            assert a is None, name
            continue
        _assert_gradient_parity("raster " + name, a, b, t)
    vo, vctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                uncertainty=sc.uncertainty)
    vr, vsaved = ref_ops.explicit_voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1),
                                               beta=sc.beta, uncertainty=sc.uncertainty)
    vst = vctx.buffers["state"]
    assert torch.equal(vst.isect_ids, vsaved["isect_ids"]) and torch.equal(vst.flatten_ids, vsaved["flatten_ids"])
    assert torch.equal(vst.offsets, vsaved["offsets"])
    for a, b in zip(_outs(vo), _outs(vr)):
        assert torch.equal(a, b)
    w = torch.randn(_outs(vo)[0].shape, generator=gen).to(device)
    wv = (0.1 * torch.randn(w.shape, generator=gen)).to(device) if unc else None
    g = r2s.voxelize_bwd(vctx, w, wv)
    r1 = ref_ops.explicit_voxelize_bwd(vsaved, sc.means, sc.quats, sc.scales, sc.densities, sc.beta, sc.uncertainty,
                                       w, wv)
    truth = _voxel_truth(vsaved, sc, w, wv)
    for name, a, b, t in zip(FIELDS, (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty), r1, truth):
        if b is None:
            assert a is None, name
            continue
        _assert_gradient_parity("voxel " + name, a, b, t)


@needs_ref
def test_low_level_ops_match_reference_build(device):
    ref = ref_ops.load()
    sc = scenes.small_scene().to(device)
    covars, ms = low.parameter_transform_fwd(sc.quats, sc.scales)
    rc, rms = ref.parameter_transform_fwd(sc.quats, sc.scales)
    assert torch.equal(covars, rc) and torch.equal(ms, rms)
    m2, c2, radii = low.world_to_image_projection_fwd(sc.means, covars, sc.viewmats, sc.Ks, 64, 64, 1e-8, 3.0)
    rm2, rc2, rradii = ref.world_to_image_projection_fwd(sc.means, covars, sc.viewmats, sc.Ks, 64, 64, 1e-8, 3.0)
    assert torch.equal(m2, rm2) and torch.equal(radii, rradii)
    torch.testing.assert_close(c2, rc2, atol=0, rtol=0)
    con, mu = low.conics_mu_fwd(c2, 1e-8)
    rcon, rmu = ref.conics_mu_fwd(c2, 1e-8)
    assert torch.equal(con, rcon) and torch.equal(mu, rmu)
    tpg, ids, fids = low.isect_tiles(m2, radii, 16, 4, 4)
    rtpg, rids, rfids = ref.isect_tiles(m2, radii, 16, 4, 4)
    assert torch.equal(tpg, rtpg) and torch.equal(ids, rids) and torch.equal(fids, rfids)
    assert torch.equal(low.isect_offset_encode(ids, 4, 4, 4), ref.isect_offset_encode(ids, 4, 4, 4))
    mv, cv, rv = low.world_to_volume_mapping_fwd(sc.means, covars, ms, sc.means.new_ones(3), sc.means.new_zeros(3),
                                                 32, 32, 32, 1e-8, 3.0)
    rmv, rcv, rrv = ref.world_to_volume_mapping_fwd(sc.means, covars, ms, sc.means.new_ones(3),
                                                    sc.means.new_zeros(3), 32, 32, 32, 1e-8, 3.0)
    assert torch.equal(mv, rmv) and torch.equal(cv, rcv) and torch.equal(rv, rrv)
    vol = torch.randn(1, 20, 21, 22, generator=torch.Generator().manual_seed(1)).to(device)
    loss, tv, tvm = low.volume_loss_fwd(vol, 0.05)
    rl, rt, rtvm = ref.volume_loss_fwd(vol, 0.05)
    assert torch.equal(tvm, rtvm)
    torch.testing.assert_close(tv, rt, atol=1e-6, rtol=1e-6)
    g1 = low.volume_loss_bwd(vol, torch.ones(1, device=device), 0.05)
    assert torch.equal(g1, ref.volume_loss_bwd(vol, torch.ones(1, device=device), 0.05))


@needs_ref
def test_ct_scale_tile_lists_and_images_match_reference_build(device):
    """Full CT-scale scene (N=200k, 64 views, 512^2, 256^3): tile lists and outputs bit for bit."""
    sc = scenes.ct_scene().to(device)
    img, ctx = r2s.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size)
    ref_img, saved = ref_ops.explicit_rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size)
    st = ctx.buffers["state"]
    assert st.n_isects == saved["isect_ids"].numel() > 1_000_000
    assert torch.equal(st.isect_ids, saved["isect_ids"])
    assert torch.equal(st.flatten_ids, saved["flatten_ids"])
    assert torch.equal(st.offsets, saved["offsets"])
    assert bool((st.isect_ids[1:] >= st.isect_ids[:-1]).all())
    assert torch.equal(img, ref_img)
    del ctx, saved
    vol, vctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1))
    ref_vol, vsaved = ref_ops.explicit_voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1))
    vst = vctx.buffers["state"]
    assert torch.equal(vst.isect_ids, vsaved["isect_ids"]) and torch.equal(vst.flatten_ids, vsaved["flatten_ids"])
    assert torch.equal(vst.offsets, vsaved["offsets"])
    assert torch.equal(vol, ref_vol)


@needs_ref
def test_ct_scale_gradients_match_reference_build(device):
    """Full CT-scale gradients (record-parallel raster VJP, voxel VJP) against the reference build.

    Unit-variance adjoints keep every gradient far above the 1e-6 absolute
    floor, so the relative 1e-5 term is what is tested.
    """
    sc = scenes.ct_scene().to(device)
    img, ctx = r2s.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size)
    _, saved = ref_ops.explicit_rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size)
    gen = torch.Generator().manual_seed(21)
    v = torch.randn(img.shape, generator=gen).to(device)
    g = r2s.rasterize_bwd(ctx, v)
    r1 = ref_ops.explicit_rasterize_bwd(saved, sc.means, sc.quats, sc.scales, None, None, v)
    truth = _raster_truth(saved, sc, v, None)
    report = {}
    for name, a, b, t in zip(FIELDS, (g.means, g.quats, g.scales, g.densities), r1, truth):
        _assert_gradient_parity("raster " + name, a, b, t, report)
    del ctx, saved, r1, truth
    vol, vctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1))
    _, vsaved = ref_ops.explicit_voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1))
    w = torch.randn(vol.shape, generator=gen).to(device)
    g = r2s.voxelize_bwd(vctx, w)
    r1 = ref_ops.explicit_voxelize_bwd(vsaved, sc.means, sc.quats, sc.scales, sc.densities, None, None, w)
    truth = _voxel_truth(vsaved, sc, w, None)
    for name, a, b, t in zip(FIELDS, (g.means, g.quats, g.scales, g.densities), r1, truth):
        _assert_gradient_parity("voxel " + name, a, b, t, report)
    print("CT-scale gradient parity:", report)


@needs_ref
@pytest.mark.parametrize("detach", [False, True])
def test_beta_uncertainty_full_scale_matches_reference_build(device, detach):
    """The 500k-primitive Beta scene with uncertainty (128 views at 768^2, volume 384^3), the
    variance branch attached or detached: 2D tile lists through the two 6-bit passes of the
    segmented sort (2,304 tiles per camera) and 3D lists bit for bit; mean and variance images
    and volumes bit for bit; all six gradients of both passes under the gradient parity check."""
    sc = scenes.beta_scene().to(device)
    gen = torch.Generator().manual_seed(1)
    c, (h, w_) = sc.viewmats.shape[0], sc.image_size
    v = torch.randn((c, h, w_), generator=gen).to(device)
    vv = (0.1 * torch.randn((c, h, w_), generator=gen)).to(device)
    out, ctx = r2s.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                 uncertainty=sc.uncertainty, detach_variance=detach)
    ref_out, saved = ref_ops.explicit_rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                                    uncertainty=sc.uncertainty)
    st = ctx.buffers["state"]
    assert st.offsets.shape[1] * st.offsets.shape[2] == 2304
    assert st.n_isects == saved["isect_ids"].numel() > 100_000_000
    assert torch.equal(st.isect_ids, saved["isect_ids"])
    assert torch.equal(st.flatten_ids, saved["flatten_ids"])
    assert torch.equal(st.offsets, saved["offsets"])
    for a, b in zip(out, ref_out):
        assert torch.equal(a, b)
    del out, ref_out
    g = r2s.rasterize_bwd(ctx, v, vv)
    r1 = ref_ops.explicit_rasterize_bwd(saved, sc.means, sc.quats, sc.scales, sc.beta, sc.uncertainty, v, vv, detach)
    truth = _raster_truth(saved, sc, v, vv, detach)
    report = {}
    for name, a, b, t in zip(FIELDS, (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty), r1, truth):
        _assert_gradient_parity("raster " + name, a, b, t, report)
    del ctx, saved, r1, truth, v, vv
    torch.cuda.empty_cache()
    w = torch.randn(sc.volume_shape, generator=gen).to(device)
    wv = (0.1 * torch.randn(sc.volume_shape, generator=gen)).to(device)
    vo, vctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                uncertainty=sc.uncertainty, detach_variance=detach)
    vr, vsaved = ref_ops.explicit_voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                               uncertainty=sc.uncertainty)
    vst = vctx.buffers["state"]
    assert torch.equal(vst.isect_ids, vsaved["isect_ids"]) and torch.equal(vst.flatten_ids, vsaved["flatten_ids"])
    assert torch.equal(vst.offsets, vsaved["offsets"])
    for a, b in zip(vo, vr):
        assert torch.equal(a, b)
    g = r2s.voxelize_bwd(vctx, w, wv)
    r1 = ref_ops.explicit_voxelize_bwd(vsaved, sc.means, sc.quats, sc.scales, sc.densities, sc.beta, sc.uncertainty,
                                       w, wv, detach)
    truth = _voxel_truth(vsaved, sc, w, wv, detach)
    for name, a, b, t in zip(FIELDS, (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty), r1, truth):
        _assert_gradient_parity("voxel " + name, a, b, t, report)
    print(f"Beta full-scale gradient parity (detach={detach}):", report)


@pytest.mark.parametrize("beta,unc,detach", [(False, False, False), (True, True, False), (True, True, True)])
def test_voxel_vjp_deterministic_and_list_free_form_agrees(device, beta, unc, detach):
    """The explicit voxel VJP gives the same bits on every run; the list-free record-parallel form (used when a
    backward keeps no intersection lists) agrees with it to fp32 summation order."""
    from r2splat_b200 import _fused

    if beta:
        sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(device)
    else:
        sc = scenes.small_scene().to(device)
    if not unc:
        sc.uncertainty = None
    gen = torch.Generator().manual_seed(31)
    w = torch.randn(sc.volume_shape, generator=gen).to(device)
    wv = (0.1 * torch.randn(sc.volume_shape, generator=gen)).to(device) if unc else None
    runs = []
    for _ in range(2):
        _, vctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                   uncertainty=sc.uncertainty, detach_variance=detach)
        g = r2s.voxelize_bwd(vctx, w, wv)
        runs.append([getattr(g, f) for f in FIELDS])
    for a, b in zip(*runs):
        assert (a is None and b is None) or torch.equal(a, b)
    extent, center = sc.means.new_ones(3), sc.means.new_zeros(3)
    radius_clip = 1.0 if beta else 3.0
    state = _fused.voxel_vjp_state(*sc.primitives, sc.volume_shape, extent, center, sc.beta, sc.uncertainty, 1e-8,
                                   radius_clip)
    assert state.offsets is None and state.n_items > 0
    lean = _fused.voxel_backward(state, sc.means, sc.quats, sc.scales, sc.beta, sc.uncertainty, extent, center, 1e-8,
                                 w, wv, detach)
    for name, a, b in zip(FIELDS, lean, runs[0]):
        if b is None:
            continue
        scale = float(b.abs().max())
        torch.testing.assert_close(a, b, rtol=1e-4, atol=1e-5 * scale, msg=name)


@pytest.mark.parametrize("beta", [False, True])
def test_released_lists_give_the_same_gradients(device, beta):
    """Freeing the forward's intersection lists before the backward (recompute-in-backward under a memory
    budget): the raster VJP never reads them, the voxel VJP switches to its list-free form."""
    from r2splat_b200 import explicit

    if beta:
        sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(device)
    else:
        sc = scenes.small_scene().to(device)
        sc.uncertainty = None
    gen = torch.Generator().manual_seed(41)
    results = []
    for release in (False, True):
        out, ctx = r2s.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                     uncertainty=sc.uncertainty)
        vo, vctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                    uncertainty=sc.uncertainty)
        if release:
            explicit.release_intersection_lists(ctx)
            explicit.release_intersection_lists(vctx)
            assert "isect_ids" not in ctx.buffers and ctx.buffers["state"].isect_ids is None
        gen.manual_seed(41)
        adj = [torch.randn(o.shape, generator=gen).to(device) for o in _outs(out)]
        vadj = [torch.randn(o.shape, generator=gen).to(device) for o in _outs(vo)]
        results.append((r2s.rasterize_bwd(ctx, *adj), r2s.voxelize_bwd(vctx, *vadj)))
    (g0, v0), (g1, v1) = results
    for name in FIELDS:
        a, b = getattr(g0, name), getattr(g1, name)
        assert (a is None and b is None) or torch.equal(a, b), name
        a, b = getattr(v0, name), getattr(v1, name)
        if a is not None:
            torch.testing.assert_close(b, a, rtol=1e-4, atol=1e-5 * float(a.abs().max()), msg=name)


@pytest.mark.parametrize("shape", [(2, 33, 40, 48), (1, 20, 21, 22), (1, 64, 64, 256)])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_tv_forward_backward_in_one_pass_equals_the_two_calls(device, shape, dtype):
    """r2s_volume_loss_fwd_bwd: map and gradient bit for bit those of volume_loss_fwd + volume_loss_bwd
    (the vectorised form for fp32 rows of whole float4s, the scalar form otherwise)."""
    vol = torch.randn(shape, generator=torch.Generator().manual_seed(12), dtype=dtype).to(device)
    g = torch.full((1,), 0.7, dtype=dtype, device=device)
    loss, tv, tv_map = low.volume_loss_fwd(vol, 0.05)
    grad = low.volume_loss_bwd(vol, g, 0.05)
    loss2, tv2, grad2, map2 = low.volume_loss_fwd_bwd(vol, g, 0.05, with_map=True)
    assert torch.equal(map2, tv_map)
    assert torch.equal(grad2, grad)
    torch.testing.assert_close(tv2, tv, rtol=1e-6, atol=0)
    torch.testing.assert_close(loss2, loss, rtol=1e-6, atol=0)
    loss3, _, grad3 = low.volume_loss_fwd_bwd(vol, g, 0.05)
    assert torch.equal(grad3, grad) and torch.equal(loss3, loss2)
