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


def _equal(a, b):
    """Each step's kernels are deterministic: the same steps give the same parameters bit for bit."""
    for x, y in zip(a, b):
        assert torch.equal(x, y)


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
    _equal(_raw(a1.scene), _raw(a2.scene))
    assert torch.equal(a1.scene.loss, a2.scene.loss)


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
    _equal(_raw(graphed.recons["x"].scene), _raw(scene))


def test_admission_by_budget(device):
    probe = serve.FitServer(budget_bytes=64 << 30, slots=2, device=device)
    probe.admit("p", _factory(device, 31))
    full = probe.recons["p"].footprint
    lean_probe = serve.FitServer(budget_bytes=64 << 30, slots=2, device=device)
    lean_probe.admit("q", lambda: batched.make_synthetic_scene(1500, 3, 48, 24, seed=31, device=device, lean=True))
    lean_fp, reserve = lean_probe.recons["q"].footprint, lean_probe.lean_reserve
    assert not lean_probe.recons["q"].graphed and reserve > 0
    # Room for one full footprint plus one lean reconstruction and its reserved transient, but (the reserve
    # being held back from the start) not for a second full footprint.
    budget = full + lean_fp + reserve + (64 << 10)
    assert full > lean_fp + (64 << 10)
    server = serve.FitServer(budget_bytes=budget, slots=2, device=device, lean_reserve_bytes=reserve)
    assert server.admit("g", _factory(device, 32))
    assert server.recons["g"].graphed
    assert server.admit("l", _factory(device, 33))  # no room for a second full footprint: lean
    assert not server.recons["l"].graphed
    assert server.lean_reserve > 0
    assert server.used + server.lean_reserve <= server.budget
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


def test_graphed_overflow_grows_capacity_and_applies_the_update(device):
    """A graphed reconstruction whose lists outgrow their capacity: the served request still applies one update."""
    server = serve.FitServer(budget_bytes=8 << 30, slots=2, device=device)
    server.admit("o", _factory(device, 51))
    recon = server.recons["o"]
    scene = recon.scene
    m2, m3 = scene.needs_capacity()
    assert m2 > 1024 and m3 > 1024  # so that 1024-entry lists overflow
    recon.graph = None
    scene.set_capacity(0, 0)  # the minimum: 1024 entries each
    server._capture(recon, warm=False)
    before = _raw(scene)
    count = int(scene.step_count.item())
    stats = server.serve([(0.0, "o")])
    assert stats.completed == 1 and stats.regrown == 1
    assert int(scene.step_count.item()) == count + 1
    assert scene.capacity_2d >= m2 and scene.capacity_3d >= m3
    assert any(not torch.equal(a, b) for a, b in zip(before, _raw(scene)))
    stats = server.serve([(0.0, "o"), (0.0005, "o")])
    assert stats.completed == 2 and stats.regrown == 0
    assert int(scene.step_count.item()) == count + 3


def test_requests_for_unadmitted_reconstructions(device):
    server = serve.FitServer(budget_bytes=8 << 30, slots=2, device=device)
    server.admit("a", _factory(device, 61))
    with pytest.raises(KeyError, match="never admitted"):
        server.serve([(0.0, "a"), (0.0, "nobody")])
    server.waiting.append(("later", _factory(device, 62)))
    stats = server.serve([(0.0, "a"), (0.0, "later"), (0.001, "a")])
    assert stats.completed == 2 and stats.rejected == 1


def test_snapshot_restore_continues_bit_identically(device):
    """A snapshot taken mid-fit and restored into a fresh reconstruction continues exactly as the original."""
    server = serve.FitServer(budget_bytes=8 << 30, slots=2, device=device)
    server.admit("s", _factory(device, 71, beta=True))
    server.serve([(0.0, "s"), (0.0, "s")])
    snap = server.snapshot("s")
    server.serve([(0.0, "s")] * 3)
    original = _raw(server.recons["s"].scene)
    other = serve.FitServer(budget_bytes=8 << 30, slots=2, device=device)
    other.admit("s", _factory(device, 71, beta=True))  # same shapes; its own warm-up step is overwritten
    other.restore("s", snap)
    assert other.recons["s"].steps == snap["steps"]
    other.serve([(0.0, "s")] * 3)
    _equal(_raw(other.recons["s"].scene), original)
    scene = other.recons["s"].scene
    assert int(scene.step_count.item()) == int(server.recons["s"].scene.step_count.item())
    with pytest.raises(ValueError):
        bad = dict(snap["state"])
        bad["means"] = bad["means"][:-1]
        scene.load_state_dict(bad)
