"""Pins the CPU oracle against the reference's golden vectors and known answers (no GPU)."""

import json
import math

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import dense, losses, tiles
from r2splat_b200._beta import beta_path_log_grad, beta_path_ratio

NAMES = ("means", "quats", "scales", "densities", "beta", "uncertainty")


def _dense_cases():
    return torch.load(GOLDEN / "dense_oracle.pt", weights_only=False)


@pytest.mark.parametrize("index", range(12))
def test_dense_oracle_matches_reference_oracle_outputs_and_vjps(index):
    case = _dense_cases()[index]
    inputs = case["inputs"]
    leaves = {k: inputs[k].clone().requires_grad_(True) for k in NAMES if k in inputs}
    prims = [leaves[k] for k in NAMES[:4]]
    options = dict(beta=leaves.get("beta"), uncertainty=leaves.get("uncertainty"), eps=0.01,
                   detach_variance=case["detach"])
    if case["op"] == "rasterize":
        out = dense.rasterize_dense(*prims, inputs["viewmats"], inputs["Ks"], (14, 20), **options)
    else:
        out = dense.voxelize_dense(*prims, (5, 7, 9), volume_extent=(1.4, 1.6, 1.8),
                                   volume_center=(0.0, 0.05, -0.05), **options)
    outs = out if isinstance(out, tuple) else (out,)
    assert len(outs) == len(case["outputs"])
    for got, want in zip(outs, case["outputs"]):
        torch.testing.assert_close(got.detach(), want, atol=1e-12, rtol=1e-10)
    loss = sum((o * a).sum() for o, a in zip(outs, case["adjoints"]))
    keys = [k for k in NAMES if k in leaves]
    grads = torch.autograd.grad(loss, [leaves[k] for k in keys], allow_unused=True)
    for key, got in zip(keys, grads):
        got = torch.zeros_like(leaves[key]) if got is None else got
        torch.testing.assert_close(got, case["grads"][key], atol=1e-10, rtol=1e-9, msg=key)


def test_oracle_covariance_is_scale_rotation_product():
    q = torch.tensor([[2.0, 0.0, 0.0, 0.0], [0.3, -0.4, 0.2, 0.5]], dtype=torch.float64)
    s = torch.tensor([[0.1, 0.2, 0.3], [0.4, 0.5, 0.6]], dtype=torch.float64)
    cov = dense.covariance_matrix(q, s)
    torch.testing.assert_close(cov[0], torch.diag(s[0].square()))
    eig = torch.linalg.eigvalsh(cov[1])
    torch.testing.assert_close(eig, s[1].square().sort().values)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_tile_oracle_matches_reference_3d_tile_bound_cases(dtype):
    spec = json.loads((GOLDEN / "tile_bounds_3d.json").read_text())
    grid = spec["grid"]
    assert len(spec["cases"]) == 12
    for case in spec["cases"]:
        means = np.asarray([case["mean"]], dtype=dtype)
        radii = np.full((1, 3), case["radius"], dtype=np.int32)
        counts, ids, fids = tiles.isect_tiles_3d(means, radii, grid["tile"], grid["tiles_x"], grid["tiles_y"],
                                                 grid["tiles_z"])
        assert counts.tolist() == [len(case["expected_ids"])], case["id"]
        assert ids.tolist() == case["expected_ids"], case["id"]
        assert fids.tolist() == [0] * len(case["expected_ids"])
        offsets = tiles.offset_encode(ids, 24)
        expected = np.searchsorted(np.asarray(case["expected_ids"], dtype=np.int64), np.arange(24))
        assert offsets.tolist() == expected.tolist()


def test_tile_oracle_2d_orders_ids_within_a_tile_and_counts_rectangles():
    means2d = np.array([[[8.0, 8.0], [20.0, 8.0], [8.0, 8.0]]], dtype=np.float32)
    radii = np.array([[[4, 4], [9, 2], [1, 1]]], dtype=np.int32)
    counts, ids, fids = tiles.isect_tiles_2d(means2d, radii, 16, 3, 2)
    assert counts.tolist() == [[1, 2, 1]]
    assert ids.tolist() == [0, 0, 0, 1]
    assert fids.tolist() == [0, 1, 2, 1]
    assert tiles.offset_encode(ids, 6).tolist() == [0, 3, 4, 4, 4, 4]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_beta_path_factor_matches_160_digit_references(dtype):
    spec = json.loads((GOLDEN / "beta_references.json").read_text())
    data = torch.tensor(spec["rows"], dtype=dtype)
    gamma = data[:, 0].clone().requires_grad_()
    ratio = beta_path_ratio(gamma)
    automatic = torch.autograd.grad(ratio.log().sum(), gamma)[0]
    tol = 3e-6 if dtype == torch.float32 else 2e-12
    assert ratio.dtype == dtype
    torch.testing.assert_close(ratio, data[:, 1], atol=0, rtol=tol)
    torch.testing.assert_close(automatic, data[:, 2], atol=0, rtol=tol)
    torch.testing.assert_close(beta_path_log_grad(gamma), data[:, 2], atol=0, rtol=tol)


def test_beta_path_factor_integer_exponent_closed_forms():
    beta = torch.tensor([1.0, 2.0, 8.0], dtype=torch.float64)
    # \int_{-1}^{1} (1 - z^2)^n dz = 2 prod_{k<=n} 2k / (2k + 1).
    expected = beta.new_tensor([2 * math.prod(2 * k / (2 * k + 1) for k in range(1, n + 1)) / math.sqrt(2 * math.pi)
                                for n in (1, 2, 8)])
    torch.testing.assert_close(beta_path_ratio(beta), expected, atol=1e-12, rtol=1e-12)
    g = torch.tensor([0.8, 3.5, 9.0, 40.0], dtype=torch.float64)
    h = 1e-5
    fd = (beta_path_ratio(g + h).log() - beta_path_ratio(g - h).log()) / (2 * h)
    torch.testing.assert_close(beta_path_log_grad(g), fd, atol=1e-8, rtol=1e-8)


def test_huge_double_beta_keeps_inactive_branch_finite():
    gamma = torch.tensor([1e100], dtype=torch.float64, requires_grad=True)
    ratio = beta_path_ratio(gamma)
    grad = torch.autograd.grad(ratio.log().sum(), gamma)[0]
    assert bool(torch.isfinite(ratio).all()) and bool(torch.isfinite(grad).all())
    torch.testing.assert_close(ratio, gamma.new_tensor([7.071067811865475e-51]), atol=0, rtol=3e-14)


def test_tv_oracle_matches_reference_edge_mean():
    case = torch.load(GOLDEN / "tv_reference.pt", weights_only=False)
    loss, tv, tv_map = losses.tv_forward(case["volume"].numpy(), case["lambda"])
    assert abs(tv - float(case["tv"])) < 1e-12
    assert abs(loss - float(case["loss"])) < 1e-12
    edges = 3 * 5 * 6 + 4 * 4 * 6 + 4 * 5 * 5  # forward differences along depth, height and width
    assert abs(tv_map.sum() / edges - tv) < 1e-12
    grad = losses.tv_backward(case["volume"].numpy(), 1.0, case["lambda"])
    np.testing.assert_allclose(grad, case["grad"].numpy(), atol=1e-14)


def test_l1_oracle_forward_and_backward():
    p = np.array([[[1.0, -2.0], [3.0, 0.5]]])
    t = np.array([[[0.0, -2.0], [4.0, 1.0]]])
    loss, l1, m = losses.l1_forward(p, t, 2.0)
    assert m.tolist() == [[[1.0, 0.0], [1.0, 0.5]]]
    assert l1 == pytest.approx(0.625) and loss == pytest.approx(1.25)
    g = losses.l1_backward(p, t, [1.0], 2.0)
    assert g.tolist() == [[[0.5, 0.0], [-0.5, -0.5]]]


@pytest.mark.parametrize("beta", [None, 2.6])
def test_absgrad_oracle_is_the_sum_of_per_pixel_gradient_magnitudes(beta):
    """absgrad_dense against autograd: the per-pixel terms v_p alpha_p(mean) differentiated one by one.

    The statistic the reference's VJPs return with absgrad (RasterizeToPixelsBwd.cu:216-221,
    :459-462) is sum_p |d(v_p alpha_p) / d mean| per component, over the samples the forward
    counts; this derives it independently of the closed form the oracle writes out.
    """
    gen = torch.Generator().manual_seed(17)
    h, w = 7, 9
    means2d = torch.tensor([[[3.1, 2.7], [5.6, 4.2]]], dtype=torch.float64)
    conics = torch.tensor([[[0.30, 0.05, 0.45], [0.12, -0.03, 0.10]]], dtype=torch.float64)
    opac = torch.tensor([[1.3, 0.7]], dtype=torch.float64)
    mus = torch.tensor([[0.9, 1.4]], dtype=torch.float64)
    v = torch.randn((1, h, w), generator=gen, dtype=torch.float64)
    betas = None if beta is None else torch.tensor([[beta, beta + 0.8]], dtype=torch.float64)
    got = dense.absgrad_dense(means2d, conics, opac, mus, v, betas=betas)
    yy, xx = torch.meshgrid(torch.arange(h, dtype=torch.float64) + 0.5, torch.arange(w, dtype=torch.float64) + 0.5,
                            indexing="ij")
    want = torch.zeros(1, 2, 2, dtype=torch.float64)
    for n in range(2):
        a, b, c = conics[0, n]

        def terms(mean):
            dx, dy = xx - mean[0], yy - mean[1]
            if betas is None:
                sigma = 0.5 * (a * dx * dx + c * dy * dy) + b * dx * dy
                alpha = opac[0, n] * mus[0, n] * torch.exp(-sigma)
                valid = (sigma >= 0) & (alpha.abs() >= 1e-5)
            else:
                d2 = a * dx * dx + 2 * b * dx * dy + c * dy * dy
                hh = (1 - d2).clamp_min(1e-300)
                alpha = opac[0, n] * mus[0, n] * hh.pow(betas[0, n])
                valid = (d2 >= 0) & (d2 < 1) & (alpha.abs() >= 1e-5)
            return torch.where(valid.detach(), v[0] * alpha, torch.zeros_like(alpha)).reshape(-1)

        jac = torch.autograd.functional.jacobian(terms, means2d[0, n].clone())  # [H*W, 2]
        want[0, n] = jac.abs().sum(0)
    assert float(want.abs().max()) > 0
    torch.testing.assert_close(got, want, rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("use_beta", [False, True])
def test_dense_oracle_on_axis_projection_matches_its_closed_form(use_beta):
    """An axis-aligned primitive on the optical axis at depth 2, seen with fx = 12, fy = 10: an
    axis-aligned profile of standard deviations (6 s_x, 5 s_y) around the principal point, scaled by
    the path factor sqrt(2 pi) s_z (Gaussian) or s_z Gamma(1/2) Gamma(b + 1) / Gamma(b + 3/2) with the
    profile (1 - d^2)^(b + 1/2) (Beta); the same case as the GPU test of the explicit operators."""
    dtype = torch.float64
    means = torch.tensor([[0.0, 0.0, 2.0]], dtype=dtype)
    quats = torch.tensor([[1.0, 0.0, 0.0, 0.0]], dtype=dtype)
    scales = torch.tensor([[0.4, 0.3, 0.25]], dtype=dtype)
    density = torch.tensor([0.8], dtype=dtype)
    beta = torch.tensor([3.5], dtype=dtype) if use_beta else None
    viewmats = torch.eye(4, dtype=dtype)[None]
    Ks = torch.tensor([[[12.0, 0.0, 4.5], [0.0, 10.0, 3.5], [0.0, 0.0, 1.0]]], dtype=dtype)
    image = dense.rasterize_dense(means, quats, scales, density, viewmats, Ks, (7, 9), beta=beta, eps=0.0)
    yy, xx = torch.meshgrid(torch.arange(7, dtype=dtype) + 0.5, torch.arange(9, dtype=dtype) + 0.5, indexing="ij")
    d2 = ((xx - 4.5) / (6 * 0.4)) ** 2 + ((yy - 3.5) / (5 * 0.3)) ** 2
    if use_beta:
        log_path = math.lgamma(0.5) + math.lgamma(4.5) - math.lgamma(5.0)
        expected = 0.8 * 0.25 * math.exp(log_path) * (1 - d2).clamp_min(0) ** 4.0
    else:
        expected = 0.8 * math.sqrt(2 * math.pi) * 0.25 * torch.exp(-d2 / 2)
    expected = torch.where(expected.abs() >= 1e-5, expected, torch.zeros_like(expected))[None]
    torch.testing.assert_close(image, expected, atol=1e-13, rtol=1e-12)


@pytest.mark.parametrize("eps", [0.0, 1e-4])
def test_dense_oracle_path_factor_at_the_principal_point(eps):
    """An isotropic Gaussian of scale s on the axis, a one-pixel image at the principal point: the
    image is the path factor sqrt(2 pi (s^2 + eps)), and its s_z derivative sqrt(2 pi) s / sqrt(s^2 + eps)."""
    scale = 0.01
    means = torch.tensor([[0.0, 0.0, 2.0]], dtype=torch.float64)
    quats = torch.tensor([[1.0, 0.0, 0.0, 0.0]], dtype=torch.float64)
    scales = torch.full((1, 3), scale, dtype=torch.float64, requires_grad=True)
    Ks = torch.tensor([[[2.0, 0.0, 0.5], [0.0, 2.0, 0.5], [0.0, 0.0, 1.0]]], dtype=torch.float64)
    image = dense.rasterize_dense(means, quats, scales, torch.ones(1, dtype=torch.float64),
                                  torch.eye(4, dtype=torch.float64)[None], Ks, (1, 1), eps=eps)
    (grad,) = torch.autograd.grad(image.sum(), scales)
    assert math.isclose(float(image.detach()), math.sqrt(2 * math.pi * (scale ** 2 + eps)), rel_tol=1e-12)
    assert math.isclose(float(grad[0, 2]), math.sqrt(2 * math.pi) * scale / math.sqrt(scale ** 2 + eps),
                        rel_tol=1e-10)


def test_dense_oracle_voxel_centre_holds_the_densities():
    """Primitives centred on the single voxel of a 1^3 volume contribute their densities (Gaussian: e^0;
    Beta: (1 - 0)^b), and the variance is the q-weighted sum of their squares."""
    means = torch.tensor([[0.0, 0.0, 2.0], [0.0, 0.0, 2.0]], dtype=torch.float64)
    quats = torch.tensor([[2.0, 0.0, 0.0, 0.0], [3.0, 0.0, 0.0, 0.0]], dtype=torch.float64)
    scales = torch.tensor([[0.2, 0.3, 0.4], [0.3, 0.4, 0.5]], dtype=torch.float64)
    densities = torch.tensor([1.2, 0.8], dtype=torch.float64)
    q = torch.tensor([0.2, 0.3], dtype=torch.float64)
    for beta in (None, torch.tensor([3.5, 1.25], dtype=torch.float64)):
        volume, variance = dense.voxelize_dense(means, quats, scales, densities, (1, 1, 1), volume_extent=(1, 1, 1),
                                                volume_center=(0, 0, 2), beta=beta, uncertainty=q, eps=0.0)
        torch.testing.assert_close(volume, torch.full((1, 1, 1), 2.0, dtype=torch.float64))
        torch.testing.assert_close(variance, torch.full((1, 1, 1), 0.2 * 1.44 + 0.3 * 0.64, dtype=torch.float64))
