"""Batched (CUDA-graph) fit steps: parity with the explicit API, the Adam update, mixing, overflow.

One fit step of a FitScene is: raster forward + MSE image gradient + raster
VJP, voxel forward + TV forward/backward + voxel VJP, then the fused
activation-chain + Adam update. Images and volumes must equal the explicit
API's bit for bit (same kernels, same tile sizes), and so must the raster and
voxel gradients: both record-parallel VJPs are deterministic.
"""

import ctypes

import pytest
import torch

import r2splat_b200 as r2s
from r2splat_b200 import batched
from r2splat_b200.cuda import _backend
from r2splat_b200.cuda import _wrapper as low

pytestmark = pytest.mark.gpu


def _small(device, seed=0, beta=False, n=2000, side=64, cameras=4, volume=32):
    return batched.make_synthetic_scene(n, cameras, side, volume, beta=beta, seed=seed, device=device)


def _physical(scene):
    return (scene.means.clone(), scene.quats.clone(), scene.scales.clone(), scene.densities.clone(),
            None if scene.beta is None else scene.beta.clone())


def _raw(scene):
    out = [scene.means, scene.quats, scene.raw_scales, scene.raw_densities]
    if scene.raw_beta is not None:
        out.append(scene.raw_beta)
    return [t.clone() for t in out]


def _params_equal(a, b):
    """Every step's kernels are deterministic, so parameters after the same steps are equal bit for bit."""
    for x, y in zip(a, b):
        assert torch.equal(x, y)


@pytest.mark.parametrize("beta", [False, True])
def test_fit_step_matches_explicit_api(device, beta):
    scene = _small(device, beta=beta)
    means, quats, scales, densities, b = _physical(scene)
    scene.step()
    cfg = scene.cfg
    image, ctx = r2s.rasterize_fwd(means, quats, scales, densities, scene.viewmats, scene.Ks, cfg.image_size, beta=b)
    assert torch.equal(scene.image, image)
    v_image = 2 * (image - scene.target) / image.numel()
    g = r2s.rasterize_bwd(ctx, v_image)
    for mine, ref in zip(scene.g_raster, (g.means, g.quats, g.scales, g.densities, g.beta)):
        if ref is not None:
            assert torch.equal(mine, ref)
    volume, vctx = r2s.voxelize_fwd(means, quats, scales, densities, cfg.volume_shape,
                                    volume_extent=cfg.volume_extent, beta=b)
    assert torch.equal(scene.volume, volume)
    # The step's loss: MSE from the forward's fused epilogue plus lambda TV.
    tv = low.volume_loss_fwd(volume.unsqueeze(0), cfg.lambda_tv)[0]
    want = ((image.double() - scene.target.double()) ** 2).mean().item() + tv.item()
    assert abs(scene.loss.item() - want) <= 1e-5 * want
    g_vol = low.volume_loss_bwd(volume.unsqueeze(0), torch.ones(1, device=device), cfg.lambda_tv)[0]
    assert torch.equal(scene.g_volume, g_vol)
    gv = r2s.voxelize_bwd(vctx, g_vol)
    for mine, ref in zip(scene.g_voxel, (gv.means, gv.quats, gv.scales, gv.densities, gv.beta)):
        if ref is not None:
            assert torch.equal(mine, ref)


def test_adam_activation_step_matches_torch_adam(device):
    gen = torch.Generator(device=device).manual_seed(4)
    n = 777
    raw = {
        "means": torch.randn(n, 3, device=device, generator=gen),
        "quats": torch.randn(n, 4, device=device, generator=gen),
        "raw_scales": torch.randn(n, 3, device=device, generator=gen) - 4,
        "raw_densities": torch.randn(n, device=device, generator=gen),
        "raw_beta": torch.randn(n, device=device, generator=gen),
    }
    params = {k: v.clone().requires_grad_() for k, v in raw.items()}
    opt = torch.optim.Adam(params.values(), lr=3e-3)
    mine = {k: v.clone() for k, v in raw.items()}
    scales, dens, beta = mine["raw_scales"].exp(), torch.nn.functional.softplus(mine["raw_densities"]), \
        mine["raw_beta"].exp()
    m = torch.zeros(n, 12, device=device)
    v = torch.zeros(n, 12, device=device)
    step = torch.zeros(1, dtype=torch.int32, device=device)
    for it in range(3):
        ga = [torch.randn(s, device=device, generator=gen) for s in ((n, 3), (n, 4), (n, 3), (n,), (n,))]
        gb = [torch.randn(s, device=device, generator=gen) for s in ((n, 3), (n, 4), (n, 3), (n,), (n,))]
        with torch.no_grad():
            s_phys = params["raw_scales"].exp()
            b_phys = params["raw_beta"].exp()
        params["means"].grad = ga[0] + gb[0]
        params["quats"].grad = ga[1] + gb[1]
        params["raw_scales"].grad = (ga[2] + gb[2]) * s_phys
        params["raw_densities"].grad = (ga[3] + gb[3]) * params["raw_densities"].detach().sigmoid()
        params["raw_beta"].grad = (ga[4] + gb[4]) * b_phys
        opt.step()
        ta = (ctypes.c_void_p * 5)(*[t.data_ptr() for t in ga])
        tb = (ctypes.c_void_p * 5)(*[t.data_ptr() for t in gb])
        _backend.call("r2s_adam_activation_step", 0, n, mine["means"].data_ptr(), mine["quats"].data_ptr(),
                      mine["raw_scales"].data_ptr(), mine["raw_densities"].data_ptr(), mine["raw_beta"].data_ptr(),
                      scales.data_ptr(), dens.data_ptr(), beta.data_ptr(), m.data_ptr(), v.data_ptr(), ta, tb,
                      3e-3, 0.9, 0.999, 1e-8, step.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert int(step.item()) == 3
    for k in raw:
        assert torch.allclose(mine[k], params[k].detach(), rtol=1e-5, atol=1e-6), k
    assert torch.allclose(scales, mine["raw_scales"].exp(), rtol=1e-6)
    assert torch.allclose(dens, torch.nn.functional.softplus(mine["raw_densities"]), rtol=1e-6)


def test_adam_step_skipped_on_overflow(device):
    scene = _small(device, n=500)
    before = _raw(scene)
    steps = int(scene.step_count.item())
    ta = (ctypes.c_void_p * 5)(*[None if t is None else t.data_ptr() for t in scene.g_raster])
    flag = torch.ones(1, dtype=torch.int32, device=device)
    _backend.call("r2s_adam_activation_step", 0, scene.n, scene.means.data_ptr(), scene.quats.data_ptr(),
                  scene.raw_scales.data_ptr(), scene.raw_densities.data_ptr(), None, scene.scales.data_ptr(),
                  scene.densities.data_ptr(), None, scene.adam_m.data_ptr(), scene.adam_v.data_ptr(), ta, None,
                  1e-3, 0.9, 0.999, 1e-8, scene.step_count.data_ptr(), flag.data_ptr(),
                  torch.cuda.current_stream().cuda_stream)
    assert int(scene.step_count.item()) == steps
    for a, b in zip(before, _raw(scene)):
        assert torch.equal(a, b)


def test_graph_replay_matches_eager_steps(device):
    eager = _small(device, seed=1)
    graphed = _small(device, seed=1)
    fit = batched.BatchedFit([graphed])
    # capture() runs one eager step per scene first; match it on the eager side.
    fit.capture()
    eager.step()
    for _ in range(3):
        fit.step()
        eager.step()
    torch.cuda.synchronize()
    assert int(graphed.step_count.item()) == int(eager.step_count.item()) == 4
    _params_equal(_raw(graphed), _raw(eager))


def test_scene_results_same_alone_and_in_a_mix(device):
    alone = batched.BatchedFit([_small(device, seed=2)])
    mix_scene = _small(device, seed=2)
    mix = batched.BatchedFit([_small(device, seed=5, n=3000, side=96, cameras=6),
                              mix_scene,
                              _small(device, seed=6, beta=True, n=1500, side=48, cameras=3, volume=24)])
    for _ in range(3):
        alone.step()
        mix.step()
    torch.cuda.synchronize()
    _params_equal(_raw(alone.scenes[0]), _raw(mix_scene))
    assert torch.equal(alone.scenes[0].loss, mix_scene.loss)


def test_capacity_overflow_is_detected_and_redone(device):
    reference = _small(device, seed=3)
    tight = _small(device, seed=3)
    fit = batched.BatchedFit([tight])
    fit.capture()  # warm-up: one real eager step
    reference.step()
    tight.set_capacity(10, 10)  # far below the real counts: the next replay must overflow
    fit.capture(warm=False)
    fit.step()  # the replay overflows; the step is redone eagerly and the graph re-captured
    reference.step()
    torch.cuda.synchronize()
    assert fit.recaptures == 1
    assert int(tight.step_count.item()) == int(reference.step_count.item()) == 2
    assert tight.capacity_2d >= int(reference.cum[-1].item())
    _params_equal(_raw(tight), _raw(reference))
    fit.step()  # the re-captured graph has room
    assert fit.recaptures == 1 and int(tight.step_count.item()) == 3


def test_autotuner_picks_a_candidate_and_caches(device):
    tuner = batched.Autotuner(steps=1)
    made = []

    def make(tile, stage_batch):
        made.append((tile, stage_batch))
        return batched.make_synthetic_scene(800, 2, 64, 16, seed=7, tile=tile, stage_batch=stage_batch,
                                            device=device)

    choice = tuner.choose(make, 800, 2, (64, 64), "gaussian")
    assert choice in made
    assert choice[0] in batched.Autotuner.TILES and choice[1] in batched.Autotuner.BATCHES
    count = len(made)
    assert tuner.choose(make, 800, 2, (64, 64), "gaussian") == choice
    assert len(made) == count
