"""Host-side logic of the serving and batched drivers (no GPU needed)."""

import pytest
import torch

from r2splat_b200 import batched, serve


def test_poisson_requests_are_sorted_seeded_and_cover_keys():
    a = serve.poisson_requests(["x", "y", "z"], rate_per_s=400.0, count=2000, seed=3)
    b = serve.poisson_requests(["x", "y", "z"], rate_per_s=400.0, count=2000, seed=3)
    assert a == b
    times = [t for t, _ in a]
    assert times == sorted(times) and times[0] > 0
    assert {k for _, k in a} == {"x", "y", "z"}
    # Mean inter-arrival time of an exponential with rate 400/s is 2.5 ms.
    assert abs(times[-1] / len(times) - 1 / 400.0) < 2e-4


def test_serve_stats_percentiles_and_summary():
    stats = serve.ServeStats(completed=5, wall_s=2.0, latencies_ms=[5.0, 1.0, 3.0, 2.0, 4.0])
    assert stats.steps_per_s == 2.5
    assert stats.percentile(50) == 3.0
    assert stats.percentile(99) == 5.0
    assert stats.percentile(0) == 1.0
    summary = stats.summary()
    assert summary["p50_ms"] == 3.0 and summary["fit_steps_per_s"] == 2.5
    assert serve.ServeStats(0, 0.0).steps_per_s == 0.0
    assert serve.ServeStats(0, 1.0).percentile(50) != serve.ServeStats(0, 1.0).percentile(50)  # nan
    assert "lean_p50_ms" not in summary


def test_serve_stats_split_lean_and_graphed_latencies():
    stats = serve.ServeStats(completed=6, wall_s=1.0, latencies_ms=[1.0, 2.0, 900.0, 3.0, 1000.0, 4.0],
                             lean_latencies_ms=[900.0, 1000.0])
    summary = stats.summary()
    assert summary["lean_requests"] == 2
    assert summary["lean_p50_ms"] in (900.0, 1000.0) and summary["lean_p99_ms"] == 1000.0
    assert summary["graphed_p99_ms"] == 4.0 and summary["graphed_p50_ms"] in (2.0, 3.0)
    assert summary["p99_ms"] == 1000.0


def test_lean_step_handle_is_done_only_when_launched_and_finished():
    from concurrent.futures import Future

    class Event:
        def __init__(self, done):
            self.done = done

        def query(self):
            return self.done

    pending = Future()
    step = serve._LeanStep(pending)
    assert not step.query()  # the worker thread has not launched it yet
    pending.set_result(Event(False))
    assert not step.query()  # launched, still running on the device
    finished = Future()
    finished.set_result(Event(True))
    assert serve._LeanStep(finished).query()
    failed = Future()
    failed.set_exception(RuntimeError("lean step failed"))
    with pytest.raises(RuntimeError, match="lean step failed"):
        serve._LeanStep(failed).query()


def test_scene_config_defaults_and_autotuner_keys():
    cfg = batched.SceneConfig(image_size=(64, 64), volume_shape=(32, 32, 32))
    assert cfg.tile == 16 and cfg.voxel_tile == 8 and cfg.stage_batch == 256 and cfg.capacity_slack > 1
    k1 = batched.Autotuner.key(100_000, 32, (512, 512), "gaussian")
    k2 = batched.Autotuner.key(120_000, 32, (512, 512), "gaussian")
    k3 = batched.Autotuner.key(100_000, 32, (512, 512), "beta")
    assert k1 == k2 and k1 != k3
    assert set(batched.Autotuner.TILES) == {8, 16, 32}


def test_mixed_benchmark_scene_shapes_follow_the_stated_distribution():
    import bench

    specs = bench._mixed_scene_specs(64, small=False)
    assert all(10_000 <= s["n"] <= 400_000 for s in specs)
    assert {s["cameras"] for s in specs} <= {16, 32, 64, 128}
    assert {s["side"] for s in specs} <= {256, 512, 1024}
    assert {s["volume"] for s in specs} <= {128, 256, 384}
    assert {s["beta"] for s in specs} == {False, True}
    assert specs == bench._mixed_scene_specs(64, small=False)
    small = bench._mixed_scene_specs(16, small=True)
    assert all(s["n"] <= 100_000 and s["side"] <= 256 for s in small)


def test_pack_roofline_counts_the_algorithmic_bytes():
    """The 3D pack pass's HBM roofline: per primitive its record, radii, first slot and slot table (written and
    read); per intersection a 4-byte id read and a 64-byte packed record written."""
    import bench

    stages = {"voxel_pack": 2.0}  # ms over two steps
    out = bench.pack_roofline(stages, 2, 1000, 10_000, 5000.0)
    nbytes = 1000 * (64 + 12 + 8 + 32) + 10_000 * 68
    assert out["algorithmic_bytes"] == nbytes and out["bound"] == "hbm"
    assert abs(out["achieved"] - nbytes / 1e-3 / 1e9) < 1e-9
    assert abs(out["frac"] - out["achieved"] / 5000.0) < 1e-12
    assert bench.pack_roofline({}, 2, 1000, 10_000, 5000.0) == {}


def test_hbm_peak_falls_back_when_the_measured_file_has_no_figure():
    """The HBM denominator is MEASURED_PEAKS.json's hbm_gbs when present; without it the bench uses the fallback
    figure and says so, instead of failing on a missing peak."""
    import bench

    assert bench.hbm_peak_gbs({"hbm_gbs": 6455.0}) == (6455.0, "MEASURED_PEAKS.json hbm_gbs")
    peak, source = bench.hbm_peak_gbs({})
    assert peak == bench.FALLBACK_HBM_GBS and source.startswith("fallback")
    out = bench.pack_roofline({"voxel_pack": 2.0}, 2, 1000, 10_000, *bench.hbm_peak_gbs({}))
    assert out["peak"] == bench.FALLBACK_HBM_GBS and out["peak_source"].startswith("fallback")
