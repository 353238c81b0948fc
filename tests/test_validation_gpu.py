"""Value checks of the explicit operators: messages, order and context behaviour.

The checks are evaluated together by one kernel (r2s_check_values); these tests
pin that each raises the reference's message (r2splat/_validation.py:35-96 and
the camera checks of r2splat/explicit.py) and that, with several problems, the
first one in the reference's order is reported, including when a host-side
check (shape, type) fails after a value check.
"""

import math

import pytest
import torch

import r2splat_b200 as r2s
from r2splat_b200 import scenes
from r2splat_b200.cuda import _backend

pytestmark = pytest.mark.gpu


def _scene(device, dtype=torch.float64, beta=False, uncertainty=False):
    sc = scenes.small_scene(dtype=dtype).to(device)
    means, quats, scales, densities = (t[:64].clone() for t in sc.primitives)
    values = {"means": means, "quats": quats, "scales": scales, "densities": densities,
              "viewmats": sc.viewmats.clone(), "Ks": sc.Ks.clone(), "image_size": (32, 32),
              "volume_shape": (16, 16, 16), "volume_extent": (1.0, 1.0, 1.0)}
    if beta:
        values["beta"] = torch.full((64,), 2.0, dtype=dtype, device=device)
    if uncertainty:
        values["uncertainty"] = torch.full((64,), 0.05, dtype=dtype, device=device)
    return values


def _raster(v):
    return r2s.rasterize_fwd(v["means"], v["quats"], v["scales"], v["densities"], v["viewmats"], v["Ks"],
                             v["image_size"], beta=v.get("beta"), uncertainty=v.get("uncertainty"))


def _voxel(v):
    return r2s.voxelize_fwd(v["means"], v["quats"], v["scales"], v["densities"], v["volume_shape"],
                            volume_extent=v["volume_extent"], beta=v.get("beta"),
                            uncertainty=v.get("uncertainty"))


def _corrupt(v, name, index, value):
    t = v[name].clone()
    t.reshape(-1)[index] = value
    v[name] = t


CASES = [
    ("means", 0, math.nan, "means must contain only finite values"),
    ("quats", 1, math.inf, "quats must contain only finite values"),
    ("scales", 2, -math.inf, "scales must contain only finite values"),
    ("densities", 3, math.nan, "densities must contain only finite values"),
    ("scales", 4, 0.0, "scales must be strictly positive physical lengths"),
    ("densities", 5, -1.0, "densities must be nonnegative"),
]


@pytest.mark.parametrize("name,index,value,message", CASES)
@pytest.mark.parametrize("operation", ["rasterize", "voxelize"])
def test_primitive_value_checks(device, operation, name, index, value, message):
    v = _scene(device)
    _corrupt(v, name, index, value)
    with pytest.raises(ValueError, match=message):
        (_raster if operation == "rasterize" else _voxel)(v)


def test_zero_quaternion_row(device):
    v = _scene(device)
    v["quats"] = v["quats"].clone()
    v["quats"][7] = 0
    with pytest.raises(ValueError, match="quats must have nonzero norm"):
        _raster(v)


@pytest.mark.parametrize("name,value,message", [
    ("beta", 0.0, "beta must contain positive 3D exponents"),
    ("beta", math.nan, "beta must contain only finite values"),
    ("uncertainty", -0.5, "uncertainty must be nonnegative relative variance"),
])
def test_optional_primitive_checks(device, name, value, message):
    v = _scene(device, beta=True, uncertainty=True)
    _corrupt(v, name, 9, value)
    with pytest.raises(ValueError, match=message):
        _raster(v)


@pytest.mark.parametrize("index,value,message", [
    (0, 0.0, "Ks must have positive fx and fy"),
    (4, -3.0, "Ks must have positive fx and fy"),
    (1, 0.5, "Ks must be pinhole intrinsics"),
    (8, 2.0, "Ks must be pinhole intrinsics"),
    (2, math.nan, "Ks must contain only finite values"),
])
def test_camera_intrinsics_checks(device, index, value, message):
    v = _scene(device)
    v["Ks"] = v["Ks"].clone()
    v["Ks"][1].reshape(-1)[index] = value
    with pytest.raises(ValueError, match=message):
        _raster(v)


def test_viewmat_last_row(device):
    v = _scene(device)
    v["viewmats"] = v["viewmats"].clone()
    v["viewmats"][2, 3, 1] = 1e-3
    with pytest.raises(ValueError, match="viewmats must have homogeneous last row"):
        _raster(v)


def test_volume_extent_positive(device):
    v = _scene(device)
    v["volume_extent"] = (1.0, 0.0, 1.0)
    with pytest.raises(ValueError, match="volume_extent must contain positive physical lengths"):
        _voxel(v)


def test_first_failure_in_reference_order(device):
    # scales <= 0 is checked before densities < 0, both after every finiteness check.
    v = _scene(device)
    _corrupt(v, "densities", 0, -1.0)
    _corrupt(v, "scales", 0, 0.0)
    with pytest.raises(ValueError, match="scales must be strictly positive"):
        _raster(v)
    # A finiteness failure of densities precedes the range check of scales.
    _corrupt(v, "densities", 1, math.nan)
    with pytest.raises(ValueError, match="densities must contain only finite values"):
        _raster(v)


def test_value_failure_before_a_later_host_failure(device):
    v = _scene(device)
    _corrupt(v, "means", 0, math.nan)
    v["quats"] = v["quats"][:10]  # a shape error, checked after means' values
    with pytest.raises(ValueError, match="means must contain only finite values"):
        _raster(v)
    v = _scene(device)
    v["quats"] = v["quats"][:10]
    with pytest.raises(ValueError, match="quats must have shape"):
        _raster(v)


@pytest.mark.parametrize("operation", ["rasterize", "voxelize"])
def test_nonfinite_adjoint_keeps_context(device, operation):
    v = _scene(device)
    output, context = (_raster if operation == "rasterize" else _voxel)(v)
    bad = output.clone()
    bad.reshape(-1)[3] = math.nan
    backward = getattr(r2s, operation + "_bwd")
    name = "v_image" if operation == "rasterize" else "v_volume"
    with pytest.raises(ValueError, match=f"{name} must contain only finite values"):
        backward(context, bad)
    grads = backward(context, torch.ones_like(output))
    assert bool(torch.isfinite(grads.densities).all())


def test_check_kernel_flags_each_kind(device):
    # Direct C-ABI call: one check per kind, bits set exactly for the failing ones.
    from r2splat_b200._validation import (FINITE, FOCAL, HOMOGENEOUS_ROW, NONNEGATIVE, PINHOLE, POSITIVE,
                                          ZERO_ROW4, _ValueCheck)
    f = torch.float32
    good = {
        FINITE: torch.ones(1000, dtype=f, device=device),
        ZERO_ROW4: torch.ones(40, dtype=f, device=device),
        POSITIVE: torch.ones(50, dtype=f, device=device),
        NONNEGATIVE: torch.zeros(50, dtype=f, device=device),
        FOCAL: torch.eye(3, dtype=f, device=device).repeat(3, 1, 1),
        PINHOLE: torch.eye(3, dtype=f, device=device).repeat(3, 1, 1),
        HOMOGENEOUS_ROW: torch.eye(4, dtype=f, device=device).repeat(2, 1, 1),
    }
    bad = {k: t.clone() for k, t in good.items()}
    bad[FINITE][999] = math.inf
    bad[ZERO_ROW4][4:8] = 0
    bad[POSITIVE][10] = 0
    bad[NONNEGATIVE][49] = -1e-30
    bad[FOCAL][2, 1, 1] = 0
    bad[PINHOLE][0, 2, 2] = 0.5
    bad[HOMOGENEOUS_ROW][1, 3, 0] = 1
    size = {FINITE: 1, ZERO_ROW4: 4, POSITIVE: 1, NONNEGATIVE: 1, FOCAL: 9, PINHOLE: 9, HOMOGENEOUS_ROW: 16}
    tensors = [good[k] for k in sorted(good)] + [bad[k] for k in sorted(bad)]
    kinds = sorted(good) * 2
    table = (_ValueCheck * len(tensors))()
    for bit, (t, kind) in enumerate(zip(tensors, kinds)):
        table[bit] = _ValueCheck(t.data_ptr(), t.numel() // size[kind], kind, bit)
    flags = torch.full((1,), -1, dtype=torch.int32, device=device)
    _backend.call("r2s_check_values", 0, table, len(tensors), flags.data_ptr(),
                  torch.cuda.current_stream(device).cuda_stream)
    word = int(flags.item()) & 0xFFFFFFFF
    assert word == ((1 << 14) - 1) & ~((1 << 7) - 1)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_finite_check_vector_path_positions(device, dtype):
    # Large finiteness checks read 16-byte vectors, four in flight per thread, then the
    # remaining vectors, then a scalar tail; unaligned data takes the element loop.
    # A single non-finite value in each region, and in an unaligned view, sets its bit.
    from r2splat_b200._validation import FINITE, _ValueCheck
    n = 1184 * 256 * 4 * 4 * 3 + 1184 * 256 * 2 + 3  # unrolled strides, single vectors and a scalar tail
    per = 16 // torch.tensor([], dtype=dtype).element_size()
    base = torch.ones(n, dtype=dtype, device=device)
    positions = {"unrolled": 12345, "vectors": (n // per) * per - per - 7, "tail": n - 1}
    tensors, bits = [base], []
    for pos in positions.values():
        t = base.clone()
        t[pos] = math.nan
        tensors.append(t)
    unaligned = base.clone()
    unaligned[n // 2] = -math.inf
    views = [(t, t.numel()) for t in tensors] + [(unaligned[1:], n - 1)]
    table = (_ValueCheck * len(views))()
    for bit, (t, count) in enumerate(views):
        assert t.data_ptr() % 16 == (0 if bit < len(tensors) else t.element_size())
        table[bit] = _ValueCheck(t.data_ptr(), count, FINITE, bit)
    flags = torch.full((1,), -1, dtype=torch.int32, device=device)
    _backend.call("r2s_check_values", 0 if dtype == torch.float32 else 1, table, len(views), flags.data_ptr(),
                  torch.cuda.current_stream(device).cuda_stream)
    word = int(flags.item()) & 0xFFFFFFFF
    assert word == (1 << len(views)) - 2  # every bit but the all-finite tensor's
