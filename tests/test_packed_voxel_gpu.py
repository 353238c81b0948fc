"""Per-tile packed 3D records with bulk-staged tile kernels, against the gather form.

``r2s_voxel_pack_tile_records`` copies each sorted intersection's record into list order
(with the pair's VJP slot in the padding); ``r2s_voxel_render_packed`` and
``r2s_voxel_render_bwd_packed`` stage each tile batch with one bulk copy. They evaluate
the same samples in the same order as the gather forms (``r2s_voxel_render``,
``r2s_voxel_render_bwd_slots``, which read records through flatten_ids), so volumes,
variances and gradients must be equal bit for bit. The scenes put hundreds of records on
a tile, so every staging barrier goes through several phases.
"""

import ctypes

import pytest
import torch

from r2splat_b200 import _fused, scenes
from r2splat_b200.cuda import _backend
from r2splat_b200.cuda import _wrapper as low

pytestmark = pytest.mark.gpu


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _faults(device, clear=True):
    count = ctypes.c_uint32(0)
    _backend.call("r2s_bulk_wait_faults", device.index or 0, int(clear), ctypes.byref(count))
    return int(count.value)


def _scene(device, dtype, beta, var, n=30000, seed=5):
    means, quats, scales, dens, b, q = scenes.random_primitives(
        n, seed, 0.03, 0.3, beta_range=(0.5, 4.0) if beta else None, uncertainty_max=0.1 if var else None,
        dtype=dtype)
    return [None if t is None else t.to(device) for t in (means, quats, scales, dens, b, q)]


def _lists(device, dtype, beta, var, shape, tile):
    means, quats, scales, dens, b, q = _scene(device, dtype, beta, var)
    covars, _ = low.parameter_transform_fwd(quats, scales)
    extent = torch.ones(3, dtype=dtype, device=device)
    center = torch.zeros(3, dtype=dtype, device=device)
    clip = 1.0 if beta else 3.0
    out = _fused.voxel_intersections(means, covars, dens, b, q, extent, center, shape, 1e-8, clip, tile)
    return means.shape[0], out


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("beta,var", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("tile", [8, 6, 4])
def test_packed_forward_and_vjp_equal_gather_form(device, dtype, beta, var, tile):
    shape = (32, 24, 40)
    n, (records, offsets, isect_ids, flatten_ids, m, means_v, radii, cum) = _lists(device, dtype, beta, var, shape,
                                                                                   tile)
    depth, height, width = shape
    tx, ty, tz = _fused._voxel_tiles(shape, tile)
    assert m > 0 and int((offsets.flatten()[1:] - offsets.flatten()[:-1]).max()) > 256  # multi-batch tiles
    _faults(device)
    stream = torch.cuda.current_stream(device).cuda_stream
    d = 0 if dtype == torch.float32 else 1

    packed = _fused.pack_tile_records(records, offsets, flatten_ids, radii, cum, m, shape, tile)
    assert torch.equal(packed[:, :12], records[flatten_ids.long()][:, :12])

    vol_g = torch.empty(shape, dtype=dtype, device=device)
    vol_p = torch.full(shape, float("nan"), dtype=dtype, device=device)
    var_g = torch.empty_like(vol_g) if var else None
    var_p = torch.full(shape, float("nan"), dtype=dtype, device=device) if var else None
    _backend.call("r2s_voxel_render", d, _p(records), int(beta), _p(offsets), _p(flatten_ids), n, m, width, height,
                  depth, tile, tx, ty, tz, _p(vol_g), _p(var_g), stream)
    _backend.call("r2s_voxel_render_packed", d, _p(packed), int(beta), _p(offsets), m, None, width, height, depth,
                  tile, tx, ty, tz, _p(vol_p), _p(var_p), stream)
    assert torch.equal(vol_g, vol_p)
    if var:
        assert torch.equal(var_g, var_p)

    gen = torch.Generator(device="cpu").manual_seed(9)
    v_vol = torch.randn(shape, generator=gen, dtype=torch.float64).to(device=device, dtype=dtype)
    v_var = (0.1 * torch.randn(shape, generator=gen, dtype=torch.float64)).to(device=device, dtype=dtype) \
        if var else None
    for detach in (0, 1):
        slots_g = torch.empty((m, 12), dtype=dtype, device=device)
        slots_p = torch.empty((m, 12), dtype=dtype, device=device)
        grads_g = torch.empty((n, 16), dtype=dtype, device=device)
        grads_p = torch.full((n, 16), float("nan"), dtype=dtype, device=device)
        _backend.call("r2s_voxel_render_bwd_slots", d, _p(records), int(beta), detach, _p(offsets), _p(flatten_ids),
                      m, None, _p(means_v), _p(radii), _p(cum), _p(v_vol), _p(v_var), n, width, height, depth, tile,
                      tx, ty, tz, _p(slots_g), m, _p(grads_g), stream)
        _backend.call("r2s_voxel_render_bwd_packed", d, _p(packed), int(beta), detach, _p(offsets), m, None,
                      _p(cum), _p(v_vol), _p(v_var), n, width, height, depth, tile, tx, ty, tz, _p(slots_p), m,
                      _p(grads_p), stream)
        assert torch.equal(grads_g, grads_p)
    torch.cuda.synchronize(device)
    assert _faults(device) == 0


def test_packed_capacity_form_writes_only_the_used_entries(device):
    """Capacity-bounded step: the count lives on the device; entries past it stay untouched, and the forward
    and VJP read only the used range."""
    dtype, shape, tile = torch.float32, (32, 32, 32), 8
    n, (records, offsets, isect_ids, flatten_ids, m, means_v, radii, cum) = _lists(device, dtype, False, False,
                                                                                   shape, tile)
    depth, height, width = shape
    tx, ty, tz = _fused._voxel_tiles(shape, tile)
    capacity = m + 777
    flat_c = torch.zeros(capacity, dtype=torch.int32, device=device)
    flat_c[:m] = flatten_ids
    n_used = torch.tensor([m], dtype=torch.int64, device=device)
    packed = torch.full((capacity, 16), -3.0, dtype=dtype, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream
    ws = torch.empty(_backend.library().r2s_voxel_pack_workspace(n), dtype=torch.uint8, device=device)
    _backend.call("r2s_voxel_pack_tile_records", 0, _p(records), _p(offsets), _p(flat_c), _p(radii), _p(cum), n,
                  capacity, _p(n_used), tile, tx, ty, tz, capacity, _p(packed), _p(ws), ws.numel(), stream)
    assert bool((packed[m:] == -3.0).all())
    reference = _fused.pack_tile_records(records, offsets, flatten_ids, radii, cum, m, shape, tile)
    assert torch.equal(packed[:m], reference)
    vol_a = torch.empty(shape, dtype=dtype, device=device)
    vol_b = torch.empty(shape, dtype=dtype, device=device)
    _backend.call("r2s_voxel_render_packed", 0, _p(reference), 0, _p(offsets), m, None, width, height, depth, tile,
                  tx, ty, tz, _p(vol_a), None, stream)
    _backend.call("r2s_voxel_render_packed", 0, _p(packed), 0, _p(offsets), 0, _p(n_used), width, height, depth,
                  tile, tx, ty, tz, _p(vol_b), None, stream)
    assert torch.equal(vol_a, vol_b)
    # Slots past a smaller slot capacity are marked unused (0xffffffff) and the VJP skips them.
    small = m // 2
    _backend.call("r2s_voxel_pack_tile_records", 0, _p(records), _p(offsets), _p(flatten_ids), _p(radii), _p(cum), n,
                  m, None, tile, tx, ty, tz, small, _p(packed), _p(ws), ws.numel(), stream)
    # Too small a workspace is refused before any launch.
    with pytest.raises(RuntimeError, match="workspace"):
        _backend.call("r2s_voxel_pack_tile_records", 0, _p(records), _p(offsets), _p(flatten_ids), _p(radii),
                      _p(cum), n, m, None, tile, tx, ty, tz, m, _p(packed), _p(ws), 16, stream)
    slot = packed[:m, 12].view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    assert bool(((slot < small) | (slot == 0xFFFFFFFF)).all())
    assert int((slot == 0xFFFFFFFF).sum()) == m - small
    torch.cuda.synchronize(device)
    assert _faults(device) == 0


@pytest.mark.parametrize("beta", [False, True])
def test_explicit_path_gathers_past_the_pack_budget_with_the_same_results(device, monkeypatch, beta):
    """A voxelize forward whose packed copy and VJP slots would exceed the pack budget keeps the gather
    form (tile kernels reading records through flatten_ids); volume, variance and gradients are the same
    bits as the packed form's."""
    import r2splat_b200 as r2s

    if beta:
        sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(device)
    else:
        sc = scenes.small_scene().to(device)
    gen = torch.Generator().manual_seed(12)
    adjoints = None
    results = []
    for budget in (None, 0):
        if budget is not None:
            monkeypatch.setattr(_fused, "VOXEL_PACK_BUDGET_BYTES", budget)
        out, ctx = r2s.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                    uncertainty=sc.uncertainty)
        state = ctx.buffers["state"]
        assert (state.packed is None) == (budget == 0)
        outs = out if isinstance(out, tuple) else (out,)
        if adjoints is None:
            adjoints = [torch.randn(o.shape, generator=gen).to(device) for o in outs]
        grads = r2s.voxelize_bwd(ctx, *adjoints)
        results.append((outs, grads))
    (o0, g0), (o1, g1) = results
    for a, b in zip(o0, o1):
        assert torch.equal(a, b)
    for name in ("means", "quats", "scales", "densities", "beta", "uncertainty"):
        a, b = getattr(g0, name), getattr(g1, name)
        assert (a is None and b is None) or torch.equal(a, b), name
    torch.cuda.synchronize(device)
    assert _faults(device) == 0


def test_slot_buffers_must_be_16_byte_aligned(device):
    """The slot writes and the per-primitive reduction use 16-byte vectors, so both slot entry points refuse a
    slot buffer that is not 16-byte aligned, before any launch."""
    dtype, shape, tile = torch.float32, (16, 16, 16), 8
    n, (records, offsets, isect_ids, flatten_ids, m, means_v, radii, cum) = _lists(device, dtype, False, False,
                                                                                   shape, tile)
    depth, height, width = shape
    tx, ty, tz = _fused._voxel_tiles(shape, tile)
    stream = torch.cuda.current_stream(device).cuda_stream
    v_vol = torch.ones(shape, dtype=dtype, device=device)
    grads = torch.empty((n, 16), dtype=dtype, device=device)
    backing = torch.empty(m * 12 + 4, dtype=dtype, device=device)
    misaligned = backing[1:].view(-1)  # 4 bytes past a 16-byte boundary
    assert misaligned.data_ptr() % 16 == 4
    with pytest.raises(RuntimeError, match="16-byte aligned"):
        _backend.call("r2s_voxel_render_bwd_slots", 0, _p(records), 0, 0, _p(offsets), _p(flatten_ids), m, None,
                      _p(means_v), _p(radii), _p(cum), _p(v_vol), None, n, width, height, depth, tile, tx, ty, tz,
                      _p(misaligned), m, _p(grads), stream)
    packed = _fused.pack_tile_records(records, offsets, flatten_ids, radii, cum, m, shape, tile)
    with pytest.raises(RuntimeError, match="16-byte aligned"):
        _backend.call("r2s_voxel_render_bwd_packed", 0, _p(packed), 0, 0, _p(offsets), m, None, _p(cum), _p(v_vol),
                      None, n, width, height, depth, tile, tx, ty, tz, _p(misaligned), m, _p(grads), stream)
