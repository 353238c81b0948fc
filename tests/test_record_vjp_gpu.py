"""Record-parallel raster VJP (``r2s_raster_record_bwd``) against a float64 restatement.

Each (camera, primitive) record's adjoints are sums over the pixels of its tile
rectangle, with the reference's per-sample rules (RasterizeToPixelsBwd.cu:350-563):
a sample counts when sigma >= 0 and |alpha| >= 1e-5, alpha = o mu exp(-sigma),
sigma = (a dx^2 + c dy^2) / 2 + b dx dy at pixel centres. The records here include
what the projection never makes: indefinite and negative-definite conics, negative
and tiny o mu. Such records fall back to the whole rectangle; their skipped
samples (sigma < 0, where exp(-sigma) overflows) must contribute nothing.
"""

import pytest
import torch

from r2splat_b200.cuda import _backend

pytestmark = pytest.mark.gpu

W, H, T = 64, 48, 16


def _records(device, n=96, seed=0):
    gen = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.rand(n, generator=gen, dtype=torch.float64) * (W + 8) - 4
    y = torch.rand(n, generator=gen, dtype=torch.float64) * (H + 8) - 4
    s = torch.exp(torch.randn(n, 2, generator=gen, dtype=torch.float64) * 0.5) * 2.5
    th = torch.rand(n, generator=gen, dtype=torch.float64) * 3.14159
    cth, sth = torch.cos(th), torch.sin(th)
    # Conic = inverse covariance of an ellipse with axes s rotated by th.
    ia, ib = 1 / s[:, 0] ** 2, 1 / s[:, 1] ** 2
    a = cth ** 2 * ia + sth ** 2 * ib
    c = sth ** 2 * ia + cth ** 2 * ib
    b = cth * sth * (ia - ib)
    o = torch.rand(n, generator=gen, dtype=torch.float64) * 0.9 + 0.05
    mu = torch.rand(n, generator=gen, dtype=torch.float64) * 2 + 0.1
    # Records the projection never produces.
    a[0], b[0], c[0] = 0.2, 0.5, 0.2            # indefinite
    a[1], b[1], c[1] = -0.1, 0.0, -0.2          # negative definite
    a[2], b[2], c[2] = 0.0, 0.3, 0.1            # singular, indefinite
    o[3] = -0.7                                 # negative o mu
    o[4] = 2e-6                                 # |alpha| < 1e-5 everywhere
    rec = torch.stack([x, y, a, b, c, o, mu, torch.zeros_like(x)], 1)
    return rec.float().to(device)


def _expected(rec, v):
    """float64 adjoints over every pixel of the full-image rectangle."""
    r = rec.double()
    x, y, a, b, c, o, mu = [r[:, i, None, None] for i in range(7)]
    py, px = torch.meshgrid(torch.arange(H, device=rec.device, dtype=torch.float64) + 0.5,
                            torch.arange(W, device=rec.device, dtype=torch.float64) + 0.5, indexing="ij")
    dx, dy = px - x, py - y
    sigma = 0.5 * (a * dx * dx + c * dy * dy) + b * dx * dy
    alpha = o * mu * torch.exp(-sigma.clamp(min=-80.0))
    keep = (sigma >= 0) & (alpha.abs() >= 1e-5)
    g = v.double()[None]
    vis = torch.where(keep, torch.exp(-sigma.clamp(min=-80.0)), torch.zeros_like(sigma))
    w = torch.where(keep, -g * alpha, torch.zeros_like(sigma))
    s = [(w * dx).sum((1, 2)), (w * dy).sum((1, 2)), (w * dx * dx).sum((1, 2)), (w * dx * dy).sum((1, 2)),
         (w * dy * dy).sum((1, 2)), (g * vis).sum((1, 2))]
    a, b, c, o, mu = [r[:, i] for i in range(2, 7)]
    return torch.stack([-(a * s[0] + b * s[1]), -(c * s[1] + b * s[0]), 0.5 * s[2], s[3], 0.5 * s[4], mu * s[5],
                        o * s[5], torch.zeros_like(a)], 1)


def _record_vjp(rec, v):
    """Packed FP32x2 walk for float32 inputs, the scalar walk for float64."""
    n = rec.shape[0]
    rects = torch.tensor([0, 0, (W + T - 1) // T, (H + T - 1) // T], dtype=torch.int16,
                         device=rec.device).repeat(n, 1)
    grads = torch.full((n, 8), float("nan"), device=rec.device, dtype=rec.dtype)
    dtype = 0 if rec.dtype == torch.float32 else 1
    _backend.call("r2s_raster_record_bwd", dtype, rec.data_ptr(), rects.data_ptr(), None, 0, 0, v.data_ptr(), None,
                  1, n, W, H, T, grads.data_ptr(), None, None, torch.cuda.current_stream(rec.device).cuda_stream)
    return grads


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("seed", [0, 1])
def test_record_vjp_matches_float64_with_degenerate_records(device, seed, dtype):
    rec = _records(device, seed=seed).to(dtype)
    gen = torch.Generator(device="cpu").manual_seed(seed + 10)
    v = torch.randn((H, W), generator=gen).to(device=device, dtype=dtype)
    got = _record_vjp(rec, v)
    want = _expected(rec, v)
    assert torch.isfinite(got).all()
    assert not got[4].any()  # |alpha| below the threshold everywhere
    scale = want.abs().amax(0).clamp(min=1e-12)
    err = ((got.double() - want).abs() / scale).amax(0)
    assert (err < 1e-4).all(), err.tolist()


def _expected_beta_var(rec, q, v, vv):
    """float64 Beta adjoints with the variance branch (q = 0 for a detached branch)."""
    r = rec.double()
    x, y, a, b, c, o, mu, beta = [r[:, i, None, None] for i in range(8)]
    qq = q.double()[:, None, None]
    py, px = torch.meshgrid(torch.arange(H, device=rec.device, dtype=torch.float64) + 0.5,
                            torch.arange(W, device=rec.device, dtype=torch.float64) + 0.5, indexing="ij")
    dx, dy = x - px, y - py
    d2 = a * dx * dx + 2 * b * dx * dy + c * dy * dy
    support = (d2 >= 0) & (d2 < 1)
    h = torch.where(support, 1 - d2, torch.ones_like(d2))
    vis = h ** beta
    alpha = o * mu * vis
    keep = support & (alpha.abs() >= 1e-5)
    g, gv = v.double()[None], vv.double()[None]
    v_eff = torch.where(keep, g + 2 * qq * alpha * gv, torch.zeros_like(d2))
    w = -o * mu * beta * h ** (beta - 1) * v_eff
    k = torch.where(keep, torch.ones_like(d2), torch.zeros_like(d2))
    s = [(w * dx).sum((1, 2)), (w * dy).sum((1, 2)), (w * dx * dx).sum((1, 2)), (w * dx * dy).sum((1, 2)),
         (w * dy * dy).sum((1, 2)), (v_eff * vis * k).sum((1, 2)), (v_eff * alpha * torch.log(h) * k).sum((1, 2)),
         (gv * alpha * alpha * k).sum((1, 2))]
    a, b, c, o, mu = [r[:, i] for i in range(2, 7)]
    grads = torch.stack([2 * (a * s[0] + b * s[1]), 2 * (b * s[0] + c * s[1]), s[2], 2 * s[3], s[4], mu * s[5],
                         o * s[5], s[6]], 1)
    a, b, c = [r[:, i, None, None] for i in range(2, 5)]
    absgrad = torch.stack([(2 * (a * w * dx + b * w * dy)).abs().sum((1, 2)),
                           (2 * (b * w * dx + c * w * dy)).abs().sum((1, 2))], 1)
    return grads, s[7], absgrad


@pytest.mark.parametrize("detach", [False, True])
def test_record_vjp_beta_variance_matches_float64(device, detach):
    n = 96
    rec = _records(device, n=n, seed=3)
    gen = torch.Generator(device="cpu").manual_seed(13)
    rec[:, 7] = (torch.rand(n, generator=gen) * 3.5 + 0.5).to(device)  # beta
    rec[:, 2:5] *= 0.25  # Beta supports of a few pixels: d^2 < 1
    q = (torch.rand(n, generator=gen) * 0.1).to(device)
    v = torch.randn((H, W), generator=gen).to(device)
    vv = (0.1 * torch.randn((H, W), generator=gen)).to(device)
    rects = torch.tensor([0, 0, (W + T - 1) // T, (H + T - 1) // T], dtype=torch.int16, device=device).repeat(n, 1)
    grads = torch.full((n, 8), float("nan"), device=device)
    v_unc = torch.zeros(n, device=device)
    _backend.call("r2s_raster_record_bwd", 0, rec.data_ptr(), rects.data_ptr(), q.data_ptr(), 1, int(detach),
                  v.data_ptr(), vv.data_ptr(), 1, n, W, H, T, grads.data_ptr(), None, v_unc.data_ptr(),
                  torch.cuda.current_stream(device).cuda_stream)
    want, want_unc, _ = _expected_beta_var(rec, torch.zeros_like(q) if detach else q, v, vv)
    assert torch.isfinite(grads).all() and torch.isfinite(v_unc).all()
    scale = want.abs().amax(0).clamp(min=1e-12)
    err = ((grads.double() - want).abs() / scale).amax(0)
    assert (err < 1e-4).all(), err.tolist()
    unc_scale = want_unc.abs().max().clamp(min=1e-12)
    assert ((v_unc.double() - want_unc).abs().max() / unc_scale).item() < 1e-4


@pytest.mark.parametrize("var,absgrad", [(True, False), (False, True), (True, True)])
def test_record_vjp_beta_mixed_box_sizes(device, var, absgrad):
    """Boxes from a few pixels to the whole image and an odd record count: boxes of at
    most 256 pixels are walked four records at a time by quarter warps, up to 1024 pixels
    two at a time by half warps, larger ones by the whole warp; a group short of records
    leaves lanes idle."""
    n = 77
    rec = _records(device, n=n, seed=5)
    gen = torch.Generator(device="cpu").manual_seed(21)
    rec[:, 7] = (torch.rand(n, generator=gen) * 3.5 + 0.5).to(device)  # beta
    rec[:, 2:5] *= torch.exp(torch.rand(n, 1, generator=gen) * 5 - 2.5).to(device)
    r = rec.double()
    det = r[:, 2] * r[:, 4] - r[:, 3] ** 2
    hx = torch.sqrt((r[:, 4] / det).clamp(min=0)) + 0.01
    hy = torch.sqrt((r[:, 2] / det).clamp(min=0)) + 0.01
    pd = (r[:, 2] > 0) & (r[:, 4] > 0) & (det > 0)
    area = ((2 * hx + 1) * (2 * hy + 1))[pd]
    assert int((area < 200).sum()) > 10 and int(((area > 300) & (area < 900)).sum()) > 3  # quarter and half groups
    assert int((~pd).sum()) >= 3  # not positive definite: the whole 64x48 rectangle, walked by the whole warp
    q = (torch.rand(n, generator=gen) * 0.1).to(device)
    v = torch.randn((H, W), generator=gen).to(device)
    vv = (0.1 * torch.randn((H, W), generator=gen)).to(device) if var else torch.zeros((H, W), device=device)
    rects = torch.tensor([0, 0, (W + T - 1) // T, (H + T - 1) // T], dtype=torch.int16, device=device).repeat(n, 1)
    grads = torch.full((n, 8), float("nan"), device=device)
    v_unc = torch.zeros(n, device=device)
    v_abs = torch.full((n, 2), float("nan"), device=device)
    _backend.call("r2s_raster_record_bwd", 0, rec.data_ptr(), rects.data_ptr(), q.data_ptr(), 1, 0,
                  v.data_ptr(), vv.data_ptr() if var else None, 1, n, W, H, T, grads.data_ptr(),
                  v_abs.data_ptr() if absgrad else None, v_unc.data_ptr() if var else None,
                  torch.cuda.current_stream(device).cuda_stream)
    want, want_unc, want_abs = _expected_beta_var(rec, q, v, vv)
    assert torch.isfinite(grads).all()
    scale = want.abs().amax(0).clamp(min=1e-12)
    err = ((grads.double() - want).abs() / scale).amax(0)
    assert (err < 1e-4).all(), err.tolist()
    if var:
        unc_scale = want_unc.abs().max().clamp(min=1e-12)
        assert ((v_unc.double() - want_unc).abs().max() / unc_scale).item() < 1e-4
    if absgrad:
        abs_scale = want_abs.abs().amax(0).clamp(min=1e-12)
        assert (((v_abs.double() - want_abs).abs() / abs_scale).amax(0) < 1e-4).all()
