"""Continuous-batching fit-step server: mix equals alone, admission by budget, statistics."""

import pytest
import torch

from r2splat_b200 import batched, serve

pytestmark = pytest.mark.gpu


def _factory(device, seed, n=1500, side=48, cameras=3, volume=24, beta=False):
    return lambda: batched.make_synthetic_scene(n, cameras, side, volume, beta=beta, seed=seed, device=device)


def _raw(scene):
    out = [scene.means, scene.quats, scene.raw_scales, scene.raw_densities]
    if scene.raw_beta is not None:
        out.append(scene.raw_beta)
    return [t.clone() for t in out]


def _agree(a, b, lr):
    for x, y in zip(a, b):
        diff = (x - y).abs()
        assert (diff > 1e-6 + 1e-5 * y.abs()).float().mean().item() <= 1e-3
        assert diff.max().item() <= 2.1 * lr + 1e-6


def test_served_result_same_alone_and_in_the_mix(device):
    alone = serve.FitServer(budget_bytes=8 << 30, slots=4, device=device)
    alone.admit("a", _factory(device, 11))
    mixed = serve.FitServer(budget_bytes=8 << 30, slots=4, device=device)
    mixed.admit("a", _factory(device, 11))
    mixed.admit("b", _factory(device, 12, n=4000, side=64, cameras=5, volume=32))
    mixed.admit("c", _factory(device, 13, beta=True))
    alone.serve([(0.0, "a")] * 4)
    requests = serve.poisson_requests(["a", "b", "c"], rate_per_s=2000.0, count=30, seed=3)
    requests = [r for r in requests if r[1] != "a"] + [(0.0, "a"), (0.001, "a"), (0.002, "a"), (0.003, "a")]
    stats = mixed.serve(requests)
    assert stats.completed == len(requests)
    a1, a2 = alone.recons["a"], mixed.recons["a"]
    assert a1.steps == a2.steps == 5  # one warm-up step at admission + four served
    _agree(_raw(a1.scene), _raw(a2.scene), a1.scene.cfg.lr * 5)


def test_lean_reconstruction_tracks_graphed_one(device):
    graphed = serve.FitServer(budget_bytes=8 << 30, slots=2, device=device)
    graphed.admit("x", _factory(device, 21))  # graphed, after one warm-up step
    scene = _factory(device, 21)()
    serve.FitServer._make_lean(scene)
    serve.lean_step(scene)  # the lean counterpart of the warm-up step
    lean = serve.FitServer(budget_bytes=8 << 30, slots=2, device=device)
    lean.recons["x"] = serve.Reconstruction("x", scene, graphed=False)
    graphed.serve([(0.0, "x")] * 3)
    lean.serve([(0.0, "x")] * 3)
    assert int(scene.step_count.item()) == int(graphed.recons["x"].scene.step_count.item()) == 4
    _agree(_raw(graphed.recons["x"].scene), _raw(scene), scene.cfg.lr * 4)


def test_admission_by_budget(device):
    probe = serve.FitServer(budget_bytes=64 << 30, slots=2, device=device)
    probe.admit("p", _factory(device, 31))
    full = probe.recons["p"].footprint
    server = serve.FitServer(budget_bytes=int(full * 1.5), slots=2, device=device)
    assert server.admit("g", _factory(device, 32))
    assert server.recons["g"].graphed
    assert server.admit("l", _factory(device, 33))  # no room for a second full footprint: lean
    assert not server.recons["l"].graphed
    assert server.used <= server.budget
    big = _factory(device, 34, n=200_000, side=256, cameras=16, volume=128)
    assert not server.admit("w", big)  # does not fit even lean: waits
    assert len(server.waiting) == 1
    stats = server.serve([(0.0, "g"), (0.0, "l"), (0.0005, "g")])
    assert stats.completed == 3 and stats.graphed == 1 and stats.lean == 1 and stats.waited_for_memory == 1


def test_stats_and_serial_baseline(device):
    server = serve.FitServer(budget_bytes=8 << 30, slots=3, device=device)
    for k in range(3):
        server.admit(k, _factory(device, 40 + k))
    requests = serve.poisson_requests([0, 1, 2], rate_per_s=500.0, count=24, seed=9)
    stats = server.serve(requests)
    s = stats.summary()
    assert s["completed"] == 24 and s["fit_steps_per_s"] > 0
    assert 0 < s["p50_ms"] <= s["p99_ms"]
    serial = serve.serve_serially({k: server.recons[k].scene for k in range(3)}, requests[:6])
    assert serial.completed == 6 and serial.percentile(50) > 0
