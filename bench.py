#!/usr/bin/env python
"""Benchmark: fwd+bwd Gaussian-sample evaluations per second of one CT fit step.

Workload (the CT-scale plain Gaussian scene, fp32): N=200,000 Gaussians
(means ~ U[-0.5,0.5]^3, quats ~ N(0,1)^4, scales ~ exp(N(log 0.01, 0.4)),
densities = softplus(N(0,1)), seed 0), C=64 views on a circular cone-beam
trajectory of radius 3, 512x512 detector (f=600, c=(256,256)). One fit step:
  rasterize_fwd -> v_image = 2 (image - target) / numel (target rendered once
  from means perturbed by N(0, 0.005), seed 2) -> rasterize_bwd;
  voxelize_fwd on 256^3 of extent 1 -> TV loss fwd/bwd (lambda 0.05) ->
  voxelize_bwd with the TV gradient as the upstream adjoint.
A "Gaussian-sample evaluation" is one (primitive, pixel) or (primitive, voxel)
pair inside an intersected tile: per pass, the sum over intersections of the
in-bounds pixels (voxels) of the intersection's tile. value counts the raster
and voxel forward and backward passes of a step.

Arms:
  --impl ours       this package (device-resident inputs for ``value``; the
                    public API with pinned host buffers for ``e2e``)
  --impl reference  the reference's own CUDA build (oracle/_ref, compiled
                    unmodified from the reference sources) driven through a
                    restatement of the reference's explicit.py call sequence

Under torchrun each rank runs its own replica of the workload (weak scaling,
no data-path collective); the timing is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import torch

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L2_FLUSH_BYTES = 512 << 20
FLOPS_PER_EVAL = {
    # FP32 operations per (primitive, pixel) sample of the Gaussian kernels,
    # counted from the reference formulas (RasterizeToPixelsFwd.cu:160-177,
    # RasterizeToPixelsBwd.cu:417-468), an FMA counting as two:
    # forward: offsets 2, quadratic form 8, exp argument 1 (+1 MUFU), alpha 1,
    # two threshold compares, accumulate 1 -> 16;
    # backward: forward part 14 + v_sigma 1 + mean adjoint 8 + 2 accumulates
    # + conic adjoints 11 + density / mu adjoints 6 -> 44.
    "raster_render": 16, "raster_render_bwd": 44,
}
# FP32 operations per sample of the Beta raster VJP with the variance branch in the reference's form
# (RasterizeToPixelsBwd.cu:817-1046), multiplies and adds counted separately: offsets 2, d^2 9, h 1,
# pow argument 1, alpha 1, variance terms 7, w with h^(beta - 1) 6, w dx and w dy 2, their moments 8,
# g vis 2, g alpha ln h 4.
BETA_VAR_VJP_FLOPS_PER_EVAL = 43
# Metric and workload description of each single-scene workload.
WORKLOAD_TEXT = {
    "ct": ("fwd+bwd Gaussian-sample evals/s (CT fit step: raster 64x512^2 + voxel 256^3 + TV)",
           "ct-plain-gaussian: N=200000, C=64 views R=3, 512x512 f=600, volume 256^3, TV lambda 0.05"),
    "ct4": ("fwd+bwd Gaussian-sample evals/s (CT fit step, 4 of the 64 views)",
            "ct4: the CT scene with every 16th view (4 views), 512x512, volume 256^3, TV lambda 0.05"),
    "small": ("fwd+bwd Gaussian-sample evals/s (small fit step: raster 4x64^2 + voxel 32^3 + TV)",
              "small: N=2000, C=4, 64x64, volume 32^3, TV lambda 0.05"),
    "beta8": ("fwd+bwd Beta-sample evals/s (Beta workload, 8 of the 128 views)",
              "beta8: the Beta workload with every 16th view (8 views), 768x768, volume 384^3"),
    "beta": ("fwd+bwd Beta-sample evals/s (raster 128x768^2 + voxel 384^3, mean and variance outputs)",
             "beta-uncertainty: N=500000, beta ~ U[0.5, 4], q ~ U[0, 0.1], C=128 views R=3, 768x768 f=900, "
             "volume 384^3, adjoints v ~ N(0, 1) and v_var ~ N(0, 0.1), variance branch attached"),
}
# DRAM bytes (read + write) of one record-parallel raster VJP launch at the CT
# workload, from ncu (dram__bytes_read.sum + dram__bytes_write.sum, one pass).
RASTER_VJP_TRAFFIC_BYTES = 535.5e6 + 366.9e6


# --------------------------------------------------------------------------- utilities

def dist_info():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(ms: float, world: int, device) -> float:
    """The job's time for a multi-rank measurement: the slowest rank's (identity on one rank)."""
    if world <= 1:
        return ms
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank_step: float, ranks: int, ms_per_step: float) -> float:
    """Whole-job throughput: every rank processes its own units per step (weak scaling, replicas)."""
    return units_per_rank_step * ranks / (ms_per_step * 1e-3)


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region.

    The polling process is started before the warm-up, so its start-up does not
    compete with the timed steps; ``mark(True)`` / ``mark(False)`` bracket the
    timed region and the summary keeps the samples taken inside it (or the one
    nearest to it when the region is shorter than the polling interval).
    """

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples: list[tuple[float, list[str]]] = []
        self.window = [None, None]
        self._proc = None
        self._thread = None

    def mark(self, start: bool):
        self.window[0 if start else 1] = time.monotonic()

    def __enter__(self):
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._thread = threading.Thread(target=self._read, daemon=True)
            self._thread.start()
            # Let nvidia-smi finish starting up (first sample in) before any step runs.
            deadline = time.monotonic() + 3.0
            while not self.samples and time.monotonic() < deadline and self._proc.poll() is None:
                time.sleep(0.01)
        except (OSError, ValueError):
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append((time.monotonic(), parts))

    def _timed_samples(self) -> list:
        start, end = self.window
        if start is None or end is None or not self.samples:
            return [parts for _, parts in self.samples]
        inside = [parts for t, parts in self.samples if start <= t <= end]
        if inside:
            return inside
        nearest = min(self.samples, key=lambda item: min(abs(item[0] - start), abs(item[0] - end)))
        return [nearest[1]]

    def __exit__(self, *exc):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=5)
        return False

    def summary(self) -> dict:
        clocks, maxes, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self._timed_samples():
            try:
                clocks.append(float(s[1]))
                maxes.append(float(s[2]))
            except ValueError:
                continue
            for name, flag in zip(names, s[5:9]):
                if flag.strip().lower() in ("active", "1"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(clocks) if clocks else None,
                "sm_max_mhz": max(maxes) if maxes else None, "reasons": sorted(reasons),
                "samples": len(clocks)}


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def flush_l2(buf: torch.Tensor):
    buf.add_(1.0)


def count_evals_2d(offsets: torch.Tensor, n_isects: int, height: int, width: int, tile: int) -> int:
    """Sum over intersections of the in-bounds pixels of their tile."""
    c, ty, tx = offsets.shape
    flat = offsets.reshape(-1).to(torch.int64)
    ends = torch.cat([flat[1:], flat.new_tensor([n_isects])])
    counts = (ends - flat).reshape(c, ty, tx)
    rows = torch.clamp(height - torch.arange(ty, device=offsets.device) * tile, max=tile)
    cols = torch.clamp(width - torch.arange(tx, device=offsets.device) * tile, max=tile)
    pix = rows[:, None] * cols[None, :]
    return int((counts * pix[None]).sum().item())


def count_evals_3d(offsets: torch.Tensor, n_isects: int, shape: tuple, tile: int) -> int:
    tz, ty, tx = offsets.shape
    flat = offsets.reshape(-1).to(torch.int64)
    ends = torch.cat([flat[1:], flat.new_tensor([n_isects])])
    counts = (ends - flat).reshape(tz, ty, tx)
    d, h, w = shape
    ar = lambda n, s: torch.clamp(s - torch.arange(n, device=offsets.device) * tile, max=tile)
    vox = ar(tz, d)[:, None, None] * ar(ty, h)[None, :, None] * ar(tx, w)[None, None, :]
    return int((counts * vox).sum().item())


# --------------------------------------------------------------------------- the fit step

class OursStep:
    """One fit step through this package's public explicit operators."""

    def __init__(self, scene, target, lambda_tv=0.05):
        import r2splat_b200 as r2s
        from r2splat_b200.cuda import _wrapper as low

        self.r2s, self.low = r2s, low
        self.scene, self.target, self.lam = scene, target, lambda_tv
        self.ones = torch.ones(1, device=scene.means.device)
        self.last = {}

    def __call__(self, means, quats, scales, densities):
        sc = self.scene
        image, ctx = self.r2s.rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size)
        self.last["raster_state"] = ctx.buffers["state"]
        v_image = 2 * (image - self.target) / image.numel()
        g = self.r2s.rasterize_bwd(ctx, v_image)
        volume, vctx = self.r2s.voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                             volume_extent=sc.volume_extent)
        self.last["voxel_state"] = vctx.buffers["state"]
        vol4 = volume.unsqueeze(0)
        loss, _, _ = self.low.volume_loss_fwd(vol4, self.lam)
        g_vol = self.low.volume_loss_bwd(vol4, self.ones, self.lam)[0]
        gv = self.r2s.voxelize_bwd(vctx, g_vol)
        return loss, (g.means + gv.means, g.quats + gv.quats, g.scales + gv.scales, g.densities + gv.densities)

    def eval_counts(self):
        rs, vs = self.last["raster_state"], self.last["voxel_state"]
        h, w = self.scene.image_size
        raster = count_evals_2d(rs.offsets, rs.n_isects, h, w, rs.tile_size)
        voxel = count_evals_3d(vs.offsets, vs.n_isects, vs.shape, vs.tile_size)
        return raster, voxel, rs.n_isects, vs.n_isects


class ReferenceStep:
    """The same fit step on the reference's own CUDA kernels (oracle/_ref)."""

    def __init__(self, scene, target, lambda_tv=0.05):
        from oracle import ref_ops

        self.ref_ops = ref_ops
        self.ref = ref_ops.load()
        self.scene, self.target, self.lam = scene, target, lambda_tv
        self.ones = torch.ones(1, device=scene.means.device)
        self.last = {}

    def __call__(self, means, quats, scales, densities):
        sc, ro = self.scene, self.ref_ops
        image, saved = ro.explicit_rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size)
        self.last["raster"] = saved
        v_image = 2 * (image - self.target) / image.numel()
        g = ro.explicit_rasterize_bwd(saved, means, quats, scales, None, None, v_image)
        volume, vsaved = ro.explicit_voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                                  volume_extent=sc.volume_extent)
        self.last["voxel"] = vsaved
        vol4 = volume.unsqueeze(0)
        loss, _, _ = self.ref.volume_loss_fwd(vol4, self.lam)
        g_vol = self.ref.volume_loss_bwd(vol4, self.ones, self.lam)[0]
        gv = ro.explicit_voxelize_bwd(vsaved, means, quats, scales, densities, None, None, g_vol)
        return loss, tuple(a + b for a, b in zip(g[:4], gv[:4]))

    def eval_counts(self):
        r, v = self.last["raster"], self.last["voxel"]
        h, w = self.scene.image_size
        raster = count_evals_2d(r["offsets"], r["isect_ids"].numel(), h, w, 16)
        voxel = count_evals_3d(v["offsets"], v["isect_ids"].numel(), v["shape"], 8)
        return raster, voxel, r["isect_ids"].numel(), v["isect_ids"].numel()


class _BetaAdjoints:
    """Fixed seeded adjoints of the Beta workload: v ~ N(0, 1) for the mean outputs and N(0, 0.1) for the
    variances, for the [C, H, W] images and the [D, H, W] volume."""

    def __init__(self, scene):
        device = scene.means.device
        gen = torch.Generator(device="cpu").manual_seed(1)
        c, (h, w) = scene.viewmats.shape[0], scene.image_size
        self.v_image = torch.randn((c, h, w), generator=gen).to(device)
        self.v_image_var = (0.1 * torch.randn((c, h, w), generator=gen)).to(device)
        self.v_volume = torch.randn(scene.volume_shape, generator=gen).to(device)
        self.v_volume_var = (0.1 * torch.randn(scene.volume_shape, generator=gen)).to(device)


class OursBetaStep(_BetaAdjoints):
    """Beta primitives with uncertainty through this package's explicit operators: rasterize and voxelize,
    mean and variance outputs, variance branch attached."""

    def __init__(self, scene, target=None):
        import r2splat_b200 as r2s

        super().__init__(scene)
        self.r2s, self.scene, self.last = r2s, scene, {}

    def __call__(self, means, quats, scales, densities, beta, uncertainty):
        sc = self.scene
        _, ctx = self.r2s.rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size, beta=beta,
                                        uncertainty=uncertainty)
        self.last["raster_state"] = ctx.buffers["state"]
        g = self.r2s.rasterize_bwd(ctx, self.v_image, self.v_image_var)
        _, vctx = self.r2s.voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                        volume_extent=sc.volume_extent, beta=beta, uncertainty=uncertainty)
        self.last["voxel_state"] = vctx.buffers["state"]
        gv = self.r2s.voxelize_bwd(vctx, self.v_volume, self.v_volume_var)
        grads = tuple(a + b for a, b in zip((g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty),
                                            (gv.means, gv.quats, gv.scales, gv.densities, gv.beta, gv.uncertainty)))
        return grads[3].sum(), grads

    eval_counts = OursStep.eval_counts


class ReferenceBetaStep(_BetaAdjoints):
    """The same Beta step on the reference's own CUDA kernels (oracle/_ref)."""

    def __init__(self, scene, target=None):
        from oracle import ref_ops

        super().__init__(scene)
        self.ref_ops, self.scene, self.last = ref_ops, scene, {}

    def __call__(self, means, quats, scales, densities, beta, uncertainty):
        sc, ro = self.scene, self.ref_ops
        _, saved = ro.explicit_rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size,
                                             beta=beta, uncertainty=uncertainty)
        self.last["raster"] = saved
        g = ro.explicit_rasterize_bwd(saved, means, quats, scales, beta, uncertainty, self.v_image,
                                      self.v_image_var)
        _, vsaved = ro.explicit_voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                             volume_extent=sc.volume_extent, beta=beta, uncertainty=uncertainty)
        self.last["voxel"] = vsaved
        gv = ro.explicit_voxelize_bwd(vsaved, means, quats, scales, densities, beta, uncertainty, self.v_volume,
                                      self.v_volume_var)
        grads = tuple(a + b for a, b in zip(g, gv) if a is not None and b is not None)
        return grads[3].sum(), grads

    eval_counts = ReferenceStep.eval_counts


def step_inputs(scene) -> tuple:
    """The per-step inputs of a workload: the primitives, plus beta and uncertainty when the scene has them."""
    return tuple(t for t in (*scene.primitives, scene.beta, scene.uncertainty) if t is not None)


def build_workload(device, workload: str):
    from r2splat_b200 import scenes

    if workload == "ct":
        scene = scenes.ct_scene()
    elif workload == "ct4":
        # Profiling case: the CT scene with 4 of its 64 views (same per-tile work, 1/16 of the images).
        scene = scenes.ct_scene()
        scene.viewmats, scene.Ks = scene.viewmats[::16].contiguous(), scene.Ks[::16].contiguous()
    elif workload == "small":
        scene = scenes.small_scene()
    elif workload in ("beta", "beta8"):
        # Beta primitives with uncertainty: N=500k, C=128 views, 768x768 (f=900), volume 384^3;
        # beta8 is the profiling case with every 16th view (8 views).
        scene = scenes.beta_scene()
        if workload == "beta8":
            scene.viewmats, scene.Ks = scene.viewmats[::16].contiguous(), scene.Ks[::16].contiguous()
        return scene.to(device), None
    else:
        raise SystemExit(f"unknown workload {workload}")
    scene = scene.to(device)
    target_scene = scene.to(device)
    target_scene.means = scenes.perturbed_means(scene.means)
    import r2splat_b200 as r2s

    target, _ = r2s.rasterize_fwd(*target_scene.primitives, target_scene.viewmats, target_scene.Ks,
                                  target_scene.image_size)
    return scene, target


def _probe_rate(name: str, device, ops_per_iter: float, iters: int) -> float:
    """Best-of-6 rate (ops/s) of a peak probe, timed with CUDA events."""
    import ctypes

    from r2splat_b200.cuda import _backend

    out = torch.zeros(4096, device=device)
    props = torch.cuda.get_device_properties(device)
    blocks, threads = props.multi_processor_count * 8, 256
    stream = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    best = 0.0
    for _ in range(6):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        _backend.call(name, ctypes.c_void_p(out.data_ptr()), blocks, threads, iters, stream)
        end.record()
        end.synchronize()
        ms = start.elapsed_time(end)
        best = max(best, ops_per_iter * blocks * threads * iters / (ms * 1e-3))
    return best


def fp32_peak_tflops(device) -> float:
    """Measured FP32 FMA issue peak (TFLOP/s) on this GPU: 128 FMAs = 256 flops per thread and step."""
    return _probe_rate("r2s_fp32_peak_probe", device, 256.0, 2048) / 1e12


def sfu_peak_gops(device) -> float:
    """Measured SFU ex2 issue peak (G ex2/s) on this GPU: 128 ex2 per thread and step."""
    return _probe_rate("r2s_sfu_peak_probe", device, 128.0, 512) / 1e9


def cpu_baseline(budget_s: float = 15.0) -> dict:
    """fp64 dense oracle on the host cores: raster fwd+bwd evaluations per second on a bounded sample."""
    from oracle import dense
    from r2splat_b200 import scenes

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    sc = scenes.ct_scene(dtype=torch.float64)
    view = slice(0, 1)
    n = 64
    prims = [t[:n].clone().requires_grad_(True) for t in sc.primitives]
    evals = 0
    t0 = time.perf_counter()
    reps = 0
    while True:
        img = dense.rasterize_dense(*prims, sc.viewmats[view], sc.Ks[view], sc.image_size, eps=1e-8, chunk=16)
        grads = torch.autograd.grad(img.sum(), prims)
        evals += 2 * n * sc.image_size[0] * sc.image_size[1]
        reps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    elapsed = time.perf_counter() - t0
    del grads
    rate = evals / elapsed
    # The dense oracle evaluates every (primitive, pixel) and (primitive, voxel) pair: a whole CT fit step
    # (200k primitives, 64 views x 512^2, 256^3 volume, forward + backward) is this many dense evaluations.
    full = sc.means.shape[0]
    dense_per_step = 2 * full * (sc.viewmats.shape[0] * sc.image_size[0] * sc.image_size[1] + 256 ** 3)
    return {"value": rate, "unit": "evals/s", "cores": threads, "kind": "port",
            "sample": f"float64 dense oracle (oracle/dense.py): {n} Gaussians x 1 view x 512x512, raster fwd+bwd "
                      f"(autograd), {reps} repetitions in {elapsed:.1f}s; dense evals counted",
            "extrapolated_ct_fit_step_s": dense_per_step / rate,
            "extrapolation": "not measured: dense evaluations of one full CT fit step divided by the measured rate"}


def timed_run(step, scene, steps, warmup, device, flush_buf, clocks=None):
    """Device-resident inputs; per-step CUDA events with an L2 flush between steps."""
    from r2splat_b200 import _fused

    prims = step_inputs(scene)
    for _ in range(warmup):
        step(*prims)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark(True)
    timer = _fused.StageTimer()
    total_ms = 0.0
    launches = 0
    for _ in range(steps):
        flush_l2(flush_buf)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        _fused.StageTimer.active = timer
        before = library_launches()
        start.record()
        step(*prims)
        end.record()
        launches += library_launches() - before
        _fused.StageTimer.active = None
        end.synchronize()
        total_ms += start.elapsed_time(end)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark(False)
    return total_ms, timer.totals_ms(), launches


def library_launches() -> int:
    """Kernels launched so far by this package's library (its own exact counter)."""
    from r2splat_b200.cuda import _backend

    return int(_backend.library().r2s_launch_count())


def e2e_run(step, scene, steps, warmup, device):
    """Public API with pinned host inputs copied in and gradients copied out each step."""
    host = [t.detach().cpu().pin_memory() for t in step_inputs(scene)]
    outs = None
    h2d = sum(t.numel() * t.element_size() for t in host)
    d2h = 0
    for i in range(warmup + steps):
        if i == warmup:
            torch.cuda.synchronize()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record()
        dev = [t.to(device, non_blocking=True) for t in host]
        loss, grads = step(*dev)
        if outs is None:
            outs = [torch.empty(g.shape, dtype=g.dtype, pin_memory=True) for g in grads] + [
                torch.empty((), dtype=loss.dtype, pin_memory=True)]
            d2h = sum(o.numel() * o.element_size() for o in outs)
        for o, g in zip(outs, list(grads) + [loss]):
            o.copy_(g, non_blocking=True)
    end.record()
    end.synchronize()
    return start.elapsed_time(end), h2d, d2h


def count_launches(step, scene, prefix: str) -> int:
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step(*step_inputs(scene))
        torch.cuda.synchronize()
    return sum(e.count for e in prof.key_averages() if prefix in e.key)


def _mixed_scene_specs(count: int, small: bool):
    """Scene shapes of the batched benchmark: per scene, N log-uniform in [10k, 400k], C in {16, 32, 64,
    128}, square detector side in {256, 512, 1024}, cubic volume side in {128, 256, 384}, Gaussian or Beta
    by a coin flip, seed = scene index. small: the serving shapes (N in [10k, 100k], C in {8, 16, 32},
    side in {128, 256}, volume in {64, 128}), sized so one GPU can keep up with the offered load."""
    specs = []
    for i in range(count):
        g = torch.Generator().manual_seed(i)
        lo, hi = (1e4, 1e5) if small else (1e4, 4e5)
        n = int(math.exp(math.log(lo) + (math.log(hi) - math.log(lo)) * torch.rand(1, generator=g).item()))
        cams = (8, 16, 32) if small else (16, 32, 64, 128)
        sides = (128, 256) if small else (256, 512, 1024)
        vols = (64, 128) if small else (128, 256, 384)
        pick = lambda options: options[int(torch.randint(len(options), (1,), generator=g).item())]
        specs.append({"n": n, "cameras": pick(cams), "side": pick(sides), "volume": pick(vols),
                      "beta": bool(torch.randint(2, (1,), generator=g).item()), "seed": i})
    return specs


def mixed_workload(args, device) -> dict:
    """Aggregate fit-steps/s of the batched (one CUDA graph) or served form vs the plain drop-in run
    scene by scene (explicit API + the same update), on many uneven reconstructions."""
    from r2splat_b200 import batched, serve

    small = args.workload == "serve"
    specs = _mixed_scene_specs(args.scenes, small)
    tuner = batched.Autotuner(steps=2)
    tuner.BATCHES = (256,)
    makers = []
    for spec in specs:
        def make(tile, stage_batch, spec=spec):
            return batched.make_synthetic_scene(spec["n"], spec["cameras"], spec["side"], spec["volume"],
                                                beta=spec["beta"], seed=spec["seed"], tile=tile,
                                                stage_batch=stage_batch, device=device)
        tile, stage = tuner.choose(make, spec["n"], spec["cameras"], (spec["side"], spec["side"]),
                                   "beta" if spec["beta"] else "gaussian")
        spec["tile"] = tile
        makers.append(lambda make=make, tile=tile, stage=stage: make(tile, stage))
    server = None
    if small:
        # Admission builds each reconstruction inside the budget accounting.
        server = serve.FitServer(budget_bytes=150 << 30, slots=8, device=device)
        for i, maker in enumerate(makers):
            server.admit(i, maker)
        scenes = [server.recons[i].scene for i in sorted(server.recons)]
    else:
        scenes = [maker() for maker in makers]
    torch.cuda.synchronize(device)
    # Plain: each scene's fit step through the explicit API, one scene after another.
    for scene in scenes:
        serve.lean_step(scene)
    torch.cuda.synchronize(device)
    rounds = max(1, args.steps // 4)
    start = time.perf_counter()
    for _ in range(rounds):
        for scene in scenes:
            serve.lean_step(scene)
    torch.cuda.synchronize(device)
    plain_s = (time.perf_counter() - start) / rounds
    config = {"workload": ("served" if small else "batched") + f" mix of {len(scenes)} reconstructions",
              "scenes": [{k: v for k, v in spec.items() if k != "seed"} for spec in specs]}
    result = {"metric": "aggregate fit-steps/s over uneven reconstructions", "unit": "fit-steps/s",
              "higher_is_better": True, "n_gpus": 1, "dtype": "f32", "data": "synthetic", "config": config,
              "plain_fit_steps_per_s": len(scenes) / plain_s}
    if not small:
        fit = batched.BatchedFit(scenes)
        fit.capture()
        for _ in range(args.warmup):
            fit.step()
        torch.cuda.synchronize(device)
        start_ev, end_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start_ev.record()
        for _ in range(args.steps):
            fit.step(check=False)
        end_ev.record()
        torch.cuda.synchronize(device)
        fit.step()  # one checked step: overflow handling stays exercised
        ms = start_ev.elapsed_time(end_ev) / args.steps
        result.update({"value": len(scenes) * 1e3 / ms, "ms_per_batched_step": ms, "steps": args.steps,
                       "warmup": args.warmup, "recaptures": fit.recaptures,
                       "vs_plain": len(scenes) * 1e3 / ms / result["plain_fit_steps_per_s"]})
        return result
    requests = serve.poisson_requests(list(server.recons), args.rate, args.requests, seed=1)
    served = server.serve(requests)
    serial = serve.serve_serially({k: r.scene for k, r in server.recons.items()}, requests)
    result.update({"value": served.steps_per_s, "served": served.summary(), "serial": serial.summary(),
                   "offered_rate_per_s": args.rate, "requests": args.requests,
                   "vs_serial": served.steps_per_s / serial.steps_per_s if serial.steps_per_s else None})
    return result


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--workload", choices=("ct", "ct4", "small", "beta", "beta8", "batched", "serve"), default="ct",
                        help="ct: the CT fit step (default); batched / serve: the multi-reconstruction forms")
    parser.add_argument("--scenes", type=int, default=32, help="reconstructions for --workload batched/serve")
    parser.add_argument("--requests", type=int, default=400, help="requests for --workload serve")
    parser.add_argument("--rate", type=float, default=400.0, help="Poisson request rate for --workload serve")
    parser.add_argument("--profile-only", action="store_true",
                        help="run the warm-up steps of the workload and exit (profiling driver, no timing)")
    parser.add_argument("--cpu-budget", type=float, default=15.0)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    args = parser.parse_args(argv)
    if args.warmup < 3:
        parser.error("--warmup must be at least 3")

    world, rank, local = dist_info()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if args.workload in ("batched", "serve"):
        if rank == 0:
            print(json.dumps(mixed_workload(args, device)))
        if world > 1:
            dist.destroy_process_group()
        return 0

    if args.impl == "reference":
        from oracle import ref_ops

        # The reference arm runs on rank 0 only; other ranks wait and exit.
        if world > 1 and rank != 0:
            dist.barrier()
            dist.destroy_process_group()
            return 0
        if not ref_ops.available():
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
            if world > 1:
                dist.barrier()
                dist.destroy_process_group()
            return 0

    scene, target = build_workload(device, args.workload)
    if args.workload in ("beta", "beta8"):
        step = OursBetaStep(scene) if args.impl == "ours" else ReferenceBetaStep(scene)
    else:
        step = OursStep(scene, target) if args.impl == "ours" else ReferenceStep(scene, target)
    if args.profile_only:
        for _ in range(args.warmup):
            step(*step_inputs(scene))
        torch.cuda.synchronize()
        return 0
    flush_buf = torch.zeros(L2_FLUSH_BYTES // 4, device=device)

    if world > 1 and args.impl == "ours":
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        total_ms, stages, own_launches = timed_run(step, scene, args.steps, args.warmup, device, flush_buf, clocks)
    ranks = world if args.impl == "ours" else 1
    total_ms = max_over_ranks(total_ms, ranks, device)
    ms_per_step = total_ms / args.steps
    raster_evals, voxel_evals, m2, m3 = step.eval_counts()
    evals_per_step = 2 * raster_evals + 2 * voxel_evals
    value = job_rate(evals_per_step, ranks, ms_per_step)

    e2e_ms, h2d, d2h = e2e_run(step, scene, args.steps, args.warmup, device)
    e2e_ms = max_over_ranks(e2e_ms, ranks, device)
    e2e_value = job_rate(evals_per_step, ranks, e2e_ms / args.steps)
    if args.impl == "ours":
        launches = own_launches
    else:
        launches = count_launches(step, scene, "r2splat::") * args.steps

    peaks = measured_peaks()
    result = {
        "metric": WORKLOAD_TEXT[args.workload][0],
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "fit_steps_per_s": (world if args.impl == "ours" else 1) * 1e3 / ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded scene generator, r2splat_b200/scenes.py)",
        "config": {
            "workload": WORKLOAD_TEXT[args.workload][1],
            "raster_isects": m2, "voxel_isects": m3,
            "raster_evals_per_pass": raster_evals, "voxel_evals_per_pass": voxel_evals,
            "l2": "flushed (512 MiB write) between timed steps",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "clocks": clocks.summary(),
        "e2e": {"value": e2e_value, "unit": "evals/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "stages_ms_per_step": {k: v / args.steps for k, v in stages.items()},
    }
    if args.impl == "reference":
        result["impl"] = "reference"
        result["e2e"] = {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        result["cpu_baseline"] = {
            "value": value, "unit": "evals/s", "cores": 0, "kind": "reference",
            "sample": "the reference's own CUDA kernels (compiled unmodified from its sources for sm_100a) on the "
                      "same B200, driven by its explicit.py call sequence; the reference has no CPU implementation "
                      "of these operators",
        }
    elif args.workload in ("beta", "beta8"):
        # The Beta VJP with the variance branch is bound by instruction issue (ncu: XU 15 %, issue 74 %);
        # its roofline counts the FP32 operations of the reference's per-sample form.
        kernel_ms = stages.get("raster_render_bwd", 0.0) / args.steps
        peak = fp32_peak_tflops(device)
        achieved = BETA_VAR_VJP_FLOPS_PER_EVAL * raster_evals / (kernel_ms * 1e-3) / 1e12 if kernel_ms else None
        result["roofline"] = {
            "kernel": "raster_record_bwd_kernel (record-parallel raster VJP, Beta with the variance branch)",
            "bound": "fp32",
            "work": f"algorithmic: {BETA_VAR_VJP_FLOPS_PER_EVAL} FP32 ops (and 5 MUFU) x the reference's tile samples "
                    "of one raster VJP pass; the kernel evaluates only the samples inside each record's box",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None, "traffic": None,
            "peak_source": "measured in-bench: FP32 FMA probe r2s_fp32_peak_probe",
            "sfu_peak_gex2_s_measured": sfu_peak_gops(device),
        }
    else:
        kernel = "raster_render_bwd"
        kernel_ms = stages.get(kernel, 0.0) / args.steps
        achieved = FLOPS_PER_EVAL[kernel] * raster_evals / (kernel_ms * 1e-3) / 1e12 if kernel_ms else None
        peak = fp32_peak_tflops(device)
        result["roofline"] = {
            "kernel": "raster_record_bwd_kernel (record-parallel raster VJP)",
            "bound": "fp32",
            "work": "algorithmic: 44 FP32 ops x the reference's tile samples of one raster VJP pass; the kernel "
                    "itself evaluates only the samples inside each record's conservative box",
            "achieved": achieved,
            "peak": peak,
            "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None,
            "traffic": RASTER_VJP_TRAFFIC_BYTES if args.workload == "ct" else None,
            "traffic_unit": "bytes per launch (ncu)",
            "peak_source": "measured in-bench: FP32 FMA probe r2s_fp32_peak_probe (MEASURED_PEAKS.json has no "
                           "FP32 figure)",
            "hbm_peak_gbs_measured": peaks.get("hbm_gbs"),
            "sfu_peak_gex2_s_measured": sfu_peak_gops(device),
        }
        if rank == 0 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(args.cpu_budget)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))
    return 0


if __name__ == "__main__":
    sys.exit(main())
