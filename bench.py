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
This package's arm takes the image-loss gradient from the forward's epilogue
(``explicit.rasterize_fwd_with_loss``) and the TV loss and gradient from one
pass, and issues the raster and voxel halves of the step, which share nothing
until the gradient sum, on two streams (``HalfStreams``); the reference's arm
runs its own separate passes, one after the other, as its package does.
A "Gaussian-sample evaluation" is one (primitive, pixel) or (primitive, voxel)
pair inside an intersected tile: per pass, the sum over intersections of the
in-bounds pixels (voxels) of the intersection's tile. value counts the raster
and voxel forward and backward passes of a step.

Arms:
  --impl ours       this package (device-resident inputs for ``value``; the
                    public API with pinned host buffers for ``e2e``)
  --impl reference  the reference's own code: its unmodified Python package
                    (explicit.py, _validation.py, _beta.py, cuda/_wrapper.py,
                    staged under oracle/_ref/py) on its own CUDA kernels
                    (oracle/_ref, compiled unmodified from the reference
                    sources). This process loads none of this package's native
                    code: the line lists the shared objects it mapped.

Both arms print a stage table of CUDA-event times around each public call
(``api_stages_ms_per_step``); this package's arm adds its kernel stages.

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
# FP32 operations per algorithmic sample in the reference's source form of each per-sample body:
# every add, subtract, multiply and compare counts one (no FMA contraction assumed); exp counts its
# argument multiply here and one MUFU ex2 besides.
SOURCE_FORM_OPS = {
    # RasterizeToPixelsFwd.cu:160-177: offsets 2, sigma 9, exp argument 1, alpha o mu vis 2, two
    # threshold compares 2, accumulate 1.
    "raster_render": 17,
    # RasterizeToPixelsBwd.cu:429-463: the forward part without its accumulate 16, v_sigma 1, mean
    # adjoints 8 and their accumulates 2, conic adjoints 11, density and mu adjoints 6.
    "raster_render_bwd": 44,
    # VoxelizeToVoxelsFwd.cu:180-215: offsets 3, sigma 18, exp argument 1, alpha 1, compares 2,
    # accumulate 1.
    "voxel_render": 26,
    # VoxelizeToVoxelsBwd.cu:398-432: the forward part without its accumulate 25, v_sigma 2, o vis 1,
    # density adjoint 2, conic adjoints 21, mean adjoints 22.
    "voxel_render_bwd": 73,
}
# The same bodies with FMA contraction (a multiply feeding an add counts once): 11 per raster forward and
# 30 per raster backward sample; in 3D the quadratic form has six terms, giving 21 per forward (offsets 3,
# sigma 13, exp 1, alpha 1, compares 2, accumulate 1) and 48 per backward sample (the forward part 20,
# v_sigma 1, density adjoint 1, conic adjoints 13, mean adjoints 13). The headline roofline fraction uses
# these, the lower of the two counts.
CONTRACTED_OPS = {"raster_render": 11, "raster_render_bwd": 30, "voxel_render": 21, "voxel_render_bwd": 48}
ACCUMULATE_KERNELS = {
    "raster_render": "raster_fwd_pair_kernel (tile forward, two pixels per lane)",
    "raster_render_bwd": "raster_record_bwd_kernel (record-parallel raster VJP)",
    "voxel_render": "voxel_fwd_kernel (tile forward, two rows of eight voxels per thread, bulk-staged packed records)",
    "voxel_render_bwd": ("voxel_bwd_lanes_kernel (one lane per (tile, primitive) pair walking the 8^3 tile in "
                         "lockstep, packed records)"),
}
# FP32 operations per sample of the Beta raster VJP with the variance branch in the reference's form
# (RasterizeToPixelsBwd.cu:817-1046), counted by the same rule: offsets 2, d^2 9, h 1, pow argument 1,
# alpha 1, variance terms 7, w with h^(beta - 1) 6, w dx and w dy 2, their moments 8, g vis 2,
# g alpha ln h 4.
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
# DRAM bytes (read + write) of one record-parallel raster VJP launch, from ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, one pass, one full-size launch of the
# shipped kernel, profiles/ct_fit_step_launch_list.md): 552.60 MB read, 372.58 MB written
# at the CT workload.
RASTER_VJP_TRAFFIC_BYTES = {"ct": 552.60e6 + 372.58e6}


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


# HBM copy bandwidth of an earlier STREAM-style measurement on B200, used only when
# MEASURED_PEAKS.json is absent.
FALLBACK_HBM_GBS = 6650.0


def measured_peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def hbm_peak_gbs(peaks: dict) -> tuple:
    """(HBM peak in GB/s, where it comes from): MEASURED_PEAKS.json's hbm_gbs, else the fallback."""
    if peaks.get("hbm_gbs"):
        return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    return FALLBACK_HBM_GBS, "fallback: an earlier STREAM-style copy on B200 (MEASURED_PEAKS.json absent)"


def flush_l2(buf: torch.Tensor):
    buf.add_(1.0)


class ApiStages:
    """CUDA-event times around each public call of a step, summed per call name.

    Recording only while ``active``; the events go on the current stream, so
    host time a call spends before its kernels (validation, synchronising reads
    of counts, allocation) shows up as device idle time inside its stage.
    """

    def __init__(self):
        self.active = False
        self.records: list = []

    def __call__(self, name: str):
        return _ApiStage(self, name)

    def totals_ms(self) -> dict:
        out: dict = {}
        for name, start, end in self.records:
            out[name] = out.get(name, 0.0) + start.elapsed_time(end)
        return out


class _ApiStage:
    def __init__(self, owner: ApiStages, name: str):
        self.owner, self.name, self.start = owner, name, None

    def __enter__(self):
        if self.owner.active:
            self.start = torch.cuda.Event(enable_timing=True)
            self.start.record()
        return self

    def __exit__(self, *exc):
        if self.start is not None:
            end = torch.cuda.Event(enable_timing=True)
            end.record()
            self.owner.records.append((self.name, self.start, end))
        return False


def mapped_native_libs() -> list:
    """Shared objects under this repository that this process has mapped (from /proc/self/maps)."""
    found = set()
    try:
        with open("/proc/self/maps") as maps:
            for line in maps:
                path = line.split()[-1] if len(line.split()) >= 6 else ""
                if path.endswith(".so") or ".so." in path or ".cpython-" in path:
                    p = Path(path)
                    try:
                        found.add(str(p.relative_to(ROOT)))
                    except ValueError:
                        continue
    except OSError:
        return []
    return sorted(found)


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

class HalfStreams:
    """Streams for the two independent halves of a fit step.

    The raster half (rasterize_fwd, its loss gradient, rasterize_bwd) and the voxel half
    (voxelize_fwd, TV, voxelize_bwd) share nothing until the gradient sum. With ``concurrent``
    the voxel half is issued first on a low-priority stream and the raster half on a
    high-priority one: each half's host read of its intersection count waits only for its own
    projection, and the voxel kernels fill the SMs around the raster kernels. Without it both
    halves run on the current stream in the reference's order (raster, then voxel), which is
    how the per-kernel stage timers and rooflines are taken.
    """

    def __init__(self):
        least, greatest = torch.cuda.Stream.priority_range()
        self.raster = torch.cuda.Stream(priority=greatest)
        self.voxel = torch.cuda.Stream(priority=least)
        self.concurrent = True

    def run(self, raster_fwd, raster_bwd, voxel_fwd, voxel_bwd, outputs):
        """Calls the four parts (each returning tensors the gradient sum reads) and joins them
        onto the current stream."""
        cur = torch.cuda.current_stream()
        if not self.concurrent:
            raster_fwd()
            raster_bwd()
            voxel_fwd()
            voxel_bwd()
            return
        self.raster.wait_stream(cur)
        self.voxel.wait_stream(cur)
        with torch.cuda.stream(self.voxel):
            voxel_fwd()
        with torch.cuda.stream(self.raster):
            raster_fwd()
        with torch.cuda.stream(self.voxel):
            voxel_bwd()
        with torch.cuda.stream(self.raster):
            raster_bwd()
        cur.wait_stream(self.raster)
        cur.wait_stream(self.voxel)
        for t in outputs():
            if t is not None:
                t.record_stream(cur)


class OursStep:
    """One fit step through this package's public explicit operators."""

    def __init__(self, scene, target, lambda_tv=0.05):
        import r2splat_b200 as r2s
        from r2splat_b200.cuda import _wrapper as low

        self.r2s, self.low = r2s, low
        self.scene, self.target, self.lam = scene, target, lambda_tv
        self.ones = torch.ones(1, device=scene.means.device)
        self.last = {}
        self.stages = ApiStages()
        self.streams = HalfStreams()

    def __call__(self, means, quats, scales, densities):
        sc, st = self.scene, self.stages
        out = {}

        def raster_fwd():
            with st("rasterize_fwd"):
                # The MSE image loss and its gradient (image - target) * 2 / numel come from the
                # forward's epilogue (the reference's step computes the gradient in a separate pass).
                _, ctx, v_image, _, _ = self.r2s.explicit.rasterize_fwd_with_loss(
                    means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size, self.target)
            self.last["raster_state"] = ctx.buffers["state"]
            out["raster"] = (ctx, v_image)

        def raster_bwd():
            with st("rasterize_bwd"):
                out["g"] = self.r2s.rasterize_bwd(*out.pop("raster"))

        def voxel_fwd():
            with st("voxelize_fwd"):
                volume, vctx = self.r2s.voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                                     volume_extent=sc.volume_extent)
            self.last["voxel_state"] = vctx.buffers["state"]
            with st("volume_loss_fwd_bwd"):
                # One pass: the TV term's upstream gradient (one) is known before its forward.
                loss, _, g_vol = self.low.volume_loss_fwd_bwd(volume.unsqueeze(0), self.ones, self.lam)
            out["voxel"] = (vctx, g_vol[0])
            out["loss"] = loss

        def voxel_bwd():
            with st("voxelize_bwd"):
                out["gv"] = self.r2s.voxelize_bwd(*out.pop("voxel"))

        self.streams.run(raster_fwd, raster_bwd, voxel_fwd, voxel_bwd,
                         lambda: (*_grad_fields(out["g"], 4), *_grad_fields(out["gv"], 4), out["loss"]))
        g, gv = out["g"], out["gv"]
        with st("gradient_sum"):
            grads = (g.means + gv.means, g.quats + gv.quats, g.scales + gv.scales, g.densities + gv.densities)
        return out["loss"], grads

    def eval_counts(self):
        rs, vs = self.last["raster_state"], self.last["voxel_state"]
        h, w = self.scene.image_size
        raster = count_evals_2d(rs.offsets, rs.n_isects, h, w, rs.tile_size)
        voxel = count_evals_3d(vs.offsets, vs.n_isects, vs.shape, vs.tile_size)
        return raster, voxel, rs.n_isects, vs.n_isects


def _grad_fields(g, k: int) -> tuple:
    """The first k gradient tensors of a ParameterGradients (means, quats, scales, densities, beta,
    uncertainty)."""
    return (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty)[:k]


class ReferenceStep:
    """The same fit step through the reference's own package (explicit.py) on its own kernels."""

    def __init__(self, scene, target, lambda_tv=0.05):
        from oracle import ref_ops

        self.ref = ref_ops.load_package()
        self.scene, self.target, self.lam = scene, target, lambda_tv
        self.ones = torch.ones(1, device=scene.means.device)
        self.last = {}
        self.stages = ApiStages()

    def _keep(self, key, ctx):
        # The reference's backward clears the context's buffers; keep what the eval count reads.
        self.last[key] = {"offsets": ctx.buffers["offsets"], "n_isects": ctx.buffers["isect_ids"].numel()}

    def __call__(self, means, quats, scales, densities):
        sc, r, st = self.scene, self.ref, self.stages
        with st("rasterize_fwd"):
            image, ctx = r.rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size)
        self._keep("raster", ctx)
        with st("image_loss_grad"):
            v_image = 2 * (image - self.target) / image.numel()
        with st("rasterize_bwd"):
            g = r.rasterize_bwd(ctx, v_image)
        with st("voxelize_fwd"):
            volume, vctx = r.voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                          volume_extent=sc.volume_extent)
        self._keep("voxel", vctx)
        vol4 = volume.unsqueeze(0)
        with st("volume_loss_fwd_bwd"):
            loss, _, _ = r.cuda.volume_loss_fwd(vol4, self.lam)
            g_vol = r.cuda.volume_loss_bwd(vol4, self.ones, self.lam)[0]
        with st("voxelize_bwd"):
            gv = r.voxelize_bwd(vctx, g_vol)
        with st("gradient_sum"):
            grads = (g.means + gv.means, g.quats + gv.quats, g.scales + gv.scales, g.densities + gv.densities)
        return loss, grads

    def eval_counts(self):
        r, v = self.last["raster"], self.last["voxel"]
        h, w = self.scene.image_size
        d, hh, ww = self.scene.volume_shape
        raster = count_evals_2d(r["offsets"], r["n_isects"], h, w, 16)
        voxel = count_evals_3d(v["offsets"], v["n_isects"], (d, hh, ww), 8)
        return raster, voxel, r["n_isects"], v["n_isects"]


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
        self.stages = ApiStages()
        self.streams = HalfStreams()

    def __call__(self, means, quats, scales, densities, beta, uncertainty):
        sc, st = self.scene, self.stages
        out = {}

        def raster_fwd():
            with st("rasterize_fwd"):
                _, ctx = self.r2s.rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size,
                                                beta=beta, uncertainty=uncertainty)
            self.last["raster_state"] = ctx.buffers["state"]
            out["ctx"] = ctx

        def raster_bwd():
            with st("rasterize_bwd"):
                out["g"] = self.r2s.rasterize_bwd(out.pop("ctx"), self.v_image, self.v_image_var)

        def voxel_fwd():
            with st("voxelize_fwd"):
                _, vctx = self.r2s.voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                                volume_extent=sc.volume_extent, beta=beta, uncertainty=uncertainty)
            self.last["voxel_state"] = vctx.buffers["state"]
            out["vctx"] = vctx

        def voxel_bwd():
            with st("voxelize_bwd"):
                out["gv"] = self.r2s.voxelize_bwd(out.pop("vctx"), self.v_volume, self.v_volume_var)

        self.streams.run(raster_fwd, raster_bwd, voxel_fwd, voxel_bwd,
                         lambda: (*_grad_fields(out["g"], 6), *_grad_fields(out["gv"], 6)))
        g, gv = out["g"], out["gv"]
        with st("gradient_sum"):
            grads = tuple(a + b for a, b in zip(_grad_fields(g, 6), _grad_fields(gv, 6)))
        return grads[3].sum(), grads

    eval_counts = OursStep.eval_counts


class ReferenceBetaStep(_BetaAdjoints):
    """The same Beta step through the reference's own package on its own kernels."""

    def __init__(self, scene, target=None):
        from oracle import ref_ops

        super().__init__(scene)
        self.ref, self.scene, self.last = ref_ops.load_package(), scene, {}
        self.stages = ApiStages()

    _keep = ReferenceStep._keep

    def __call__(self, means, quats, scales, densities, beta, uncertainty):
        sc, r, st = self.scene, self.ref, self.stages
        with st("rasterize_fwd"):
            _, ctx = r.rasterize_fwd(means, quats, scales, densities, sc.viewmats, sc.Ks, sc.image_size,
                                     beta=beta, uncertainty=uncertainty)
        self._keep("raster", ctx)
        with st("rasterize_bwd"):
            g = r.rasterize_bwd(ctx, self.v_image, self.v_image_var)
        with st("voxelize_fwd"):
            _, vctx = r.voxelize_fwd(means, quats, scales, densities, sc.volume_shape,
                                     volume_extent=sc.volume_extent, beta=beta, uncertainty=uncertainty)
        self._keep("voxel", vctx)
        with st("voxelize_bwd"):
            gv = r.voxelize_bwd(vctx, self.v_volume, self.v_volume_var)
        with st("gradient_sum"):
            grads = tuple(a + b for a, b in zip(
                (g.means, g.quats, g.scales, g.densities, g.beta, g.uncertainty),
                (gv.means, gv.quats, gv.scales, gv.densities, gv.beta, gv.uncertainty)))
        return grads[3].sum(), grads

    eval_counts = ReferenceStep.eval_counts


def step_inputs(scene) -> tuple:
    """The per-step inputs of a workload: the primitives, plus beta and uncertainty when the scene has them."""
    return tuple(t for t in (*scene.primitives, scene.beta, scene.uncertainty) if t is not None)


def build_workload(device, workload: str, impl: str = "ours"):
    """The workload's scene on ``device`` and, for the fit-step workloads, its target images.

    The target is rendered by the arm's own implementation, so the reference
    arm runs no code of this package's library.
    """
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
    if impl == "reference":
        from oracle import ref_ops

        api = ref_ops.load_package()
    else:
        import r2splat_b200 as api
    target, _ = api.rasterize_fwd(*target_scene.primitives, target_scene.viewmats, target_scene.Ks,
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


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as info:
            for line in info:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _config1_fit_step_cpu(sc, v_image, lam):
    """One float64 fit step of the small configuration with the dense oracle: raster fwd + bwd against
    ``v_image``, voxel fwd, TV fwd/bwd, voxel bwd with the TV gradient as its adjoint."""
    from oracle import dense, losses

    prims = [t.clone().requires_grad_(True) for t in sc.primitives]
    img = dense.rasterize_dense(*prims, sc.viewmats, sc.Ks, sc.image_size, eps=1e-8, chunk=1000)
    raster_grads = torch.autograd.grad((img * v_image).sum(), prims)
    prims = [t.detach().clone().requires_grad_(True) for t in sc.primitives]
    vol = dense.voxelize_dense(*prims, sc.volume_shape, volume_extent=sc.volume_extent, eps=1e-8, chunk=1000)
    vol_np = vol.detach().unsqueeze(0).numpy()
    losses.tv_forward(vol_np, lam)
    g_vol = torch.from_numpy(losses.tv_backward(vol_np, 1.0, lam)[0])
    voxel_grads = torch.autograd.grad((vol * g_vol).sum(), prims)
    return [a + b for a, b in zip(raster_grads, voxel_grads)]


def cpu_baseline(device, budget_s: float = 15.0) -> dict:
    """The float64 dense oracle on the host cores, run on the small configuration in full.

    Small configuration: N=2,000, C=4 views at 64x64, volume 32^3, v_image ~
    N(0, 1) (seed 1), TV lambda 0.05. ``value`` is that step's algorithmic
    evaluations (the tile samples the reference's kernels evaluate, counted on
    the GPU path) per second of host time; the oracle itself evaluates every
    (primitive, sample) pair, and ``dense_evals_per_s`` counts those.
    """
    import r2splat_b200 as r2s
    from r2splat_b200 import scenes

    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    small = scenes.small_scene()
    # Algorithmic evaluations of the small step, from the GPU path's own tile lists.
    dev = small.to(device)
    _, ctx = r2s.rasterize_fwd(*dev.primitives, dev.viewmats, dev.Ks, dev.image_size)
    _, vctx = r2s.voxelize_fwd(*dev.primitives, dev.volume_shape, volume_extent=dev.volume_extent)
    rs, vs = ctx.buffers["state"], vctx.buffers["state"]
    raster = count_evals_2d(rs.offsets, rs.n_isects, *dev.image_size, rs.tile_size)
    voxel = count_evals_3d(vs.offsets, vs.n_isects, vs.shape, vs.tile_size)
    algorithmic = 2 * raster + 2 * voxel
    sc = scenes.small_scene(dtype=torch.float64)
    c, (h, w) = sc.viewmats.shape[0], sc.image_size
    v_image = torch.randn((c, h, w), generator=torch.Generator().manual_seed(1), dtype=torch.float64)
    n = sc.means.shape[0]
    dense_per_step = 2 * n * (c * h * w + math.prod(sc.volume_shape))
    steps = 0
    t0 = time.perf_counter()
    while True:
        _config1_fit_step_cpu(sc, v_image, 0.05)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    elapsed = time.perf_counter() - t0
    dense_rate = dense_per_step * steps / elapsed
    # The CT step (N=200k, 64 views at 512^2, volume 256^3) through the same dense oracle: not run, its
    # dense evaluation count divided by the rate measured here.
    ct_dense = 2 * 200_000 * (64 * 512 * 512 + 256 ** 3)
    return {"value": algorithmic * steps / elapsed, "unit": "evals/s", "cores": threads, "kind": "port",
            "cpu_model": cpu_model(), "torch_threads": torch.get_num_threads(),
            "sample": f"small configuration in full (N=2000, 4 views at 64x64, volume 32^3, TV): {steps} float64 "
                      f"fit steps of the dense oracle (oracle/dense.py, autograd VJPs) in {elapsed:.1f} s",
            "seconds_per_fit_step": elapsed / steps,
            "algorithmic_evals_per_step": algorithmic,
            "dense_evals_per_s": dense_rate,
            "ct_step_seconds_extrapolated": ct_dense / dense_rate,
            "ct_step_extrapolation": "not measured: the CT step's 2 N (C H W + D H W) dense evaluations divided by "
                                     "dense_evals_per_s"}


def timed_run(step, scene, steps, warmup, device, flush_buf, clocks=None, ours=True):
    """Device-resident inputs; per-step CUDA events with an L2 flush between steps.

    Returns (total ms, kernel-stage ms, public-call-stage ms, launches). The
    kernel stages and this library's launch counter exist only in this
    package's arm (``ours``); the reference arm never touches the library.
    """
    prims = step_inputs(scene)
    for _ in range(warmup):
        step(*prims)
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark(True)
    timer = None
    if ours:
        from r2splat_b200 import _fused

        timer = _fused.StageTimer()
    total_ms = 0.0
    launches = 0
    per_step: list = []
    step.stages.active = True
    for _ in range(steps):
        flush_l2(flush_buf)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if ours:
            _fused.StageTimer.active = timer
            before = library_launches()
        start.record()
        step(*prims)
        end.record()
        if ours:
            launches += library_launches() - before
            _fused.StageTimer.active = None
        end.synchronize()
        per_step.append(start.elapsed_time(end))
        total_ms += per_step[-1]
    step.stages.active = False
    timed_run.per_step_ms = per_step
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark(False)
    return total_ms, (timer.totals_ms() if timer else {}), step.stages.totals_ms(), launches


def library_launches() -> int:
    """Kernels launched so far by this package's library (its own exact counter)."""
    from r2splat_b200.cuda import _backend

    return int(_backend.library().r2s_launch_count())


def e2e_run(step, scene, steps, warmup, device):
    """Public API with pinned host inputs copied in and gradients copied out each step.

    The copies run on a stream of their own, double-buffered: step i+1's inputs are copied in
    while step i computes (once step i-1, the last reader of that buffer, is done), and step
    i's gradients are copied out as soon as it ends. Every step's copies are inside the timed
    region; the clock stops when the last gradients have reached the host.
    """
    host = [t.detach().cpu().pin_memory() for t in step_inputs(scene)]
    h2d = sum(t.numel() * t.element_size() for t in host)
    cur = torch.cuda.current_stream()
    copy = torch.cuda.Stream()
    dev = [[torch.empty_like(t, device=device) for t in host] for _ in range(2)]
    loaded = [torch.cuda.Event(), torch.cuda.Event()]
    outs = None
    d2h = 0
    last_step = None
    total = warmup + steps

    def load(i):
        with torch.cuda.stream(copy):
            for d, h in zip(dev[i % 2], host):
                d.copy_(h, non_blocking=True)
            loaded[i % 2].record(copy)

    load(0)
    for i in range(total):
        if i == warmup:
            torch.cuda.synchronize()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(cur)
            copy.wait_stream(cur)
            load(i)  # this step's inputs inside the timed region
        cur.wait_event(loaded[i % 2])
        loss, grads = step(*dev[i % 2])
        done = torch.cuda.Event()
        done.record(cur)
        if i + 1 < total and i + 1 != warmup:
            if last_step is not None:
                copy.wait_event(last_step)  # the previous step read the buffer about to be overwritten
            load(i + 1)
        last_step = done
        results = list(grads) + [loss]
        if outs is None:
            outs = [[torch.empty(g.shape, dtype=g.dtype, pin_memory=True) for g in results] for _ in range(2)]
            d2h = sum(o.numel() * o.element_size() for o in outs[0])
        copy.wait_event(done)
        with torch.cuda.stream(copy):
            for o, g in zip(outs[i % 2], results):
                g.record_stream(copy)
                o.copy_(g, non_blocking=True)
    end.record(copy)
    end.synchronize()
    return start.elapsed_time(end), h2d, d2h


def count_launches(step, scene) -> dict:
    """Kernels one step launches, from the torch profiler: all of them, and those outside torch's own."""
    from torch.profiler import ProfilerActivity, profile

    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        step(*step_inputs(scene))
        torch.cuda.synchronize()
    kernels = [e for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
    own = [e for e in kernels if not any(tag in e.name for tag in ("at::", "at_cuda_detail", "Memset", "Memcpy",
                                                                    "cub::", "void at::"))]
    return {"all": len(kernels), "operator_kernels": len(own)}


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


def mixed_workload(args, device, autotune: bool = True) -> dict:
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
        if autotune:
            tile, stage = tuner.choose(make, spec["n"], spec["cameras"], (spec["side"], spec["side"]),
                                       "beta" if spec["beta"] else "gaussian")
        else:
            tile, stage = 16, 256
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
        recaptures = fit.recaptures
        del fit
        # Device work of each scene's step alone (its own one-scene graph, CUDA events): batching
        # removes host time and overlaps scenes, but cannot remove this work.
        device_ms = []
        for scene in scenes:
            one = batched.BatchedFit([scene])
            one.capture(warm=False)
            one.step(check=False)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(2):
                one.step(check=False)
            b.record()
            torch.cuda.synchronize(device)
            device_ms.append(a.elapsed_time(b) / 2)
            del one
        result.update({"value": len(scenes) * 1e3 / ms, "ms_per_batched_step": ms, "steps": args.steps,
                       "warmup": args.warmup, "recaptures": recaptures,
                       "vs_plain": len(scenes) * 1e3 / ms / result["plain_fit_steps_per_s"],
                       "plain_ms_per_round": plain_s * 1e3,
                       "sum_device_ms_per_round": sum(device_ms),
                       "host_free_bound_vs_plain": plain_s * 1e3 / sum(device_ms)})
        return result
    requests = serve.poisson_requests(list(server.recons), args.rate, args.requests, seed=1)
    served = server.serve(requests)
    serial = serve.serve_serially({k: r.scene for k, r in server.recons.items()}, requests)
    result.update({"value": served.steps_per_s, "served": served.summary(), "serial": serial.summary(),
                   "offered_rate_per_s": args.rate, "requests": args.requests,
                   "vs_serial": served.steps_per_s / serial.steps_per_s if serial.steps_per_s else None})
    return result


def _estimated_full_bytes(spec: dict) -> float:
    """Rough device footprint of a fully allocated FitScene (step buffers, lists with slack, slots and the
    per-tile packed 3D records)."""
    n, c, side, vol = spec["n"], spec["cameras"], spec["side"], spec["volume"]
    sigma_vox = 0.01 * vol
    m2 = 4.0 * c * n
    m3 = n * (6 * sigma_vox / 8 + 1) ** 3
    return (c * n * 84 + 3 * 4 * c * side * side + n * 160 + 8 * vol ** 3 + 1.3 * (12 * m2 + 124 * m3))


def serving_at_scale(args, device) -> dict:
    """The serving loop on the large mix: 200 reconstructions drawn from the 32-scene distribution (N
    log-uniform in [10k, 400k], 16-128 views, 256-1024^2, 128-384^3, Gaussian or Beta), three of them
    with N = 2,000,000 and a 1024^3 volume; a 150 GB HBM budget; reconstructions that do not fit graphed
    run lean with recompute-in-backward. Measures the saturated throughput first, then serves Poisson
    arrivals at 80 % of it and at the requested rate, against the plain drop-in run serially on the same
    requests."""
    from r2splat_b200 import batched, serve

    specs = _mixed_scene_specs(args.scenes, small=False)
    for spec in specs[:3]:
        spec.update(n=2_000_000, volume=1024)
    server = serve.FitServer(budget_bytes=150 << 30, slots=8, device=device, lean_recompute=True)
    built_lean = 0
    t0 = time.perf_counter()
    for i, spec in enumerate(specs):
        lean = _estimated_full_bytes(spec) > (16 << 30)
        built_lean += int(lean)

        def make(spec=spec, lean=lean):
            return batched.make_synthetic_scene(spec["n"], spec["cameras"], spec["side"], spec["volume"],
                                                beta=spec["beta"], seed=spec["seed"], device=device, lean=lean)
        server.admit(i, make)
    admit_s = time.perf_counter() - t0
    keys = sorted(server.recons)
    # Saturated: every request arrives at once.
    burst = [(0.0, key) for _, key in serve.poisson_requests(keys, 1.0, args.requests, seed=4)]
    saturated = server.serve(burst)
    rate_ok = 0.8 * saturated.steps_per_s
    runs = {}
    for label, rate in (("sustained", rate_ok), ("offered", args.rate)):
        requests = serve.poisson_requests(keys, rate, args.requests, seed=5)
        runs[label] = {"offered_rate_per_s": rate, "served": server.serve(requests).summary()}
    serial_requests = serve.poisson_requests(keys, rate_ok, args.requests, seed=5)
    serial = serve.serve_serially({k: server.recons[k].scene for k in keys}, serial_requests)
    return {"metric": "served fit-steps/s and p50/p99 step latency at scale", "unit": "fit-steps/s",
            "value": runs["sustained"]["served"]["fit_steps_per_s"], "higher_is_better": True, "n_gpus": 1,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{len(specs)} reconstructions (3 with N=2M, 1024^3), 150 GB budget",
                       "admitted": len(keys), "waiting": len(server.waiting), "built_lean": built_lean,
                       "graphed": sum(server.recons[k].graphed for k in keys), "admission_s": admit_s,
                       "budget_used_gb": server.used / 2**30},
            "saturated": saturated.summary(), **runs,
            "serial_at_sustained_rate": serial.summary(),
            "vs_serial": runs["sustained"]["served"]["fit_steps_per_s"] / serial.steps_per_s
            if serial.steps_per_s else None}


def bounded_mix(device, kind: str) -> dict:
    """A bounded run of the batched or served form for the default bench line.

    batched: the first 8 reconstructions of the 32-scene mix (N log-uniform in [10k, 400k], 16-128
    views, 256-1024^2, 128-384^3, Gaussian or Beta), raster tile 16 (``--workload batched`` runs all
    32 with the autotuner); served: 16 small reconstructions, 200 Poisson requests at 400/s.
    """
    ns = argparse.Namespace(workload=kind, scenes=8 if kind == "batched" else 16, steps=4, warmup=3,
                            requests=200, rate=400.0)
    out = mixed_workload(ns, device, autotune=False)
    out.pop("config", None)
    out["scenes"] = ns.scenes
    return out


def accumulate_rooflines(workload, stages, steps, raster_evals, voxel_evals, fp32_peak) -> dict:
    """Per accumulate kernel: its mean CUDA-event time per launch, and the FP32 rate its algorithmic work
    (the reference's tile samples times the per-sample operation count) represents, against the
    FP32 issue peak measured in the same run. The kernels evaluate only the samples inside each record's
    conservative box, so this is a work-equivalent rate."""
    out = {}
    beta = workload in ("beta", "beta8")
    for stage, kernel in ACCUMULATE_KERNELS.items():
        if stage not in stages or not stages[stage]:
            continue
        ms = stages[stage] / steps
        evals = raster_evals if stage.startswith("raster") else voxel_evals
        entry = {"kernel": kernel, "ms": ms, "samples": evals}
        if beta:
            if stage == "raster_render_bwd":
                entry["ops_per_sample"] = BETA_VAR_VJP_FLOPS_PER_EVAL
                entry["achieved_tflops"] = BETA_VAR_VJP_FLOPS_PER_EVAL * evals / (ms * 1e-3) / 1e12
                entry["frac"] = entry["achieved_tflops"] / fp32_peak
        else:
            ops = SOURCE_FORM_OPS[stage]
            entry["ops_per_sample_source_form"] = ops
            entry["achieved_tflops_source_form"] = ops * evals / (ms * 1e-3) / 1e12
            entry["frac_source_form"] = entry["achieved_tflops_source_form"] / fp32_peak
            if stage in CONTRACTED_OPS:
                entry["ops_per_sample_contracted"] = CONTRACTED_OPS[stage]
                entry["achieved_tflops_contracted"] = CONTRACTED_OPS[stage] * evals / (ms * 1e-3) / 1e12
                entry["frac_contracted"] = entry["achieved_tflops_contracted"] / fp32_peak
        out[stage] = entry
    return out


def pack_roofline(stages, steps, n_prims, voxel_isects, hbm_peak, peak_source="MEASURED_PEAKS.json hbm_gbs") -> dict:
    """HBM roofline of the 3D pack pass (voxel_slot_affine + pack_tile_records3 kernels): its algorithmic bytes
    read each input once (records N x 64 B, radii N x 12 B, tile-count scan N x 8 B, the slot table N x 16 B
    written and read, flatten_ids M x 4 B, offsets) and write the packed records (M x 64 B)."""
    if not stages.get("voxel_pack"):
        return {}
    ms = stages["voxel_pack"] / steps
    nbytes = n_prims * (64 + 12 + 8 + 2 * 16) + voxel_isects * (4 + 64)
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"kernel": "voxel_slot_affine_kernel + pack_tile_records3_kernel (per-tile packed 3D records)",
            "bound": "hbm", "ms": ms, "algorithmic_bytes": nbytes, "achieved": achieved, "peak": hbm_peak,
            "unit": "GB/s", "frac": achieved / hbm_peak, "peak_source": peak_source}


def dominant_roofline(workload, rooflines, fp32_peak, sfu_peak, hbm_peak) -> dict:
    """The roofline object of the step's dominant kernel, the record-parallel raster VJP."""
    entry = rooflines.get("raster_render_bwd", {})
    beta = workload in ("beta", "beta8")
    if beta:
        achieved, ops, frac = entry.get("achieved_tflops"), BETA_VAR_VJP_FLOPS_PER_EVAL, entry.get("frac")
        work = (f"algorithmic: {ops} FP32 ops (and 5 MUFU) x the reference's tile samples of one raster VJP pass "
                "(Beta with the variance branch); the kernel evaluates only the samples inside each record's box")
    else:
        achieved, frac = entry.get("achieved_tflops_contracted"), entry.get("frac_contracted")
        ops = CONTRACTED_OPS["raster_render_bwd"]
        work = (f"algorithmic: {ops} FP32 ops (FMA contracted; {SOURCE_FORM_OPS['raster_render_bwd']} in the "
                "reference's source form) x the reference's tile samples of one raster VJP pass; the kernel "
                "evaluates only the samples inside each record's conservative box")
    traffic = RASTER_VJP_TRAFFIC_BYTES.get(workload)
    return {
        "kernel": ACCUMULATE_KERNELS["raster_render_bwd"],
        "bound": "fp32",
        "work": work,
        "achieved": achieved,
        "peak": fp32_peak,
        "unit": "TFLOP/s",
        "frac": frac,
        "frac_source_form": entry.get("frac_source_form"),
        "kernel_ms": entry.get("ms"),
        "traffic": traffic,
        "traffic_unit": "DRAM bytes read + written per launch (ncu)",
        "peak_source": "measured in-bench: FP32 FMA issue probe r2s_fp32_peak_probe (MEASURED_PEAKS.json has no "
                       "FP32 figure)",
        "hbm_peak_gbs_measured": hbm_peak,
        "sfu_peak_gex2_s_measured": sfu_peak,
    }


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=20)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--workload", choices=("ct", "ct4", "small", "beta", "beta8", "batched", "serve", "serve5"),
                        default="ct",
                        help="ct: the CT fit step (default); batched / serve: the multi-reconstruction forms")
    parser.add_argument("--scenes", type=int, default=32, help="reconstructions for --workload batched/serve")
    parser.add_argument("--requests", type=int, default=400, help="requests for --workload serve")
    parser.add_argument("--rate", type=float, default=400.0, help="Poisson request rate for --workload serve")
    parser.add_argument("--profile-only", action="store_true",
                        help="run the warm-up steps of the workload and exit (profiling driver, no timing)")
    parser.add_argument("--cpu-budget", type=float, default=15.0)
    parser.add_argument("--no-cpu-baseline", action="store_true")
    parser.add_argument("--no-mix", action="store_true",
                        help="skip the bounded batched / served runs that the default CT line carries")
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
    if args.workload in ("batched", "serve", "serve5"):
        if rank == 0:
            out = serving_at_scale(args, device) if args.workload == "serve5" else mixed_workload(args, device)
            print(json.dumps(out))
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
        if not ref_ops.package_available():
            print(json.dumps({"impl": "reference",
                              "unavailable": "reference build or staged package (oracle/_ref) missing"}))
            if world > 1:
                dist.barrier()
                dist.destroy_process_group()
            return 0

    ours = args.impl == "ours"
    scene, target = build_workload(device, args.workload, args.impl)
    if args.workload in ("beta", "beta8"):
        step = OursBetaStep(scene) if ours else ReferenceBetaStep(scene)
    else:
        step = OursStep(scene, target) if ours else ReferenceStep(scene, target)
    if ours and args.workload == "small":
        # The small step is host-bound (about a millisecond): a second stream only adds host work.
        step.streams.concurrent = False
    if args.profile_only:
        for _ in range(args.warmup):
            step(*step_inputs(scene))
        torch.cuda.synchronize()
        return 0
    flush_buf = torch.zeros(L2_FLUSH_BYTES // 4, device=device)

    if world > 1 and ours:
        dist.barrier()
    torch.cuda.synchronize()
    concurrent = None
    stage_steps = args.steps
    if ours and step.streams.concurrent:
        # In the timed steps the two halves overlap, so a kernel's CUDA-event time includes the
        # other half's blocks sharing the SMs. The stage tables and rooflines are taken first, from
        # steps of the same fit step with both halves on one stream (the reference's order).
        step.streams.concurrent = False
        stage_steps = min(args.steps, 10)
        seq_ms, seq_stages, seq_api, _ = timed_run(step, scene, stage_steps, args.warmup, device, flush_buf, None,
                                                   ours=True)
        step.streams.concurrent = True
        step.stages = ApiStages()
        concurrent = {"sequential_ms_per_step": seq_ms / stage_steps}
    with ClockSampler(local) as clocks:
        total_ms, stages, api_stages, own_launches = timed_run(step, scene, args.steps, args.warmup, device,
                                                               flush_buf, clocks, ours=ours)
    per_step = sorted(getattr(timed_run, "per_step_ms", []))
    if concurrent is not None:
        concurrent.update(stages_ms_per_step={k: v / args.steps for k, v in stages.items()},
                          api_stages_ms_per_step={k: v / args.steps for k, v in api_stages.items()})
        stages, api_stages = seq_stages, seq_api
    stage_ms = concurrent["sequential_ms_per_step"] if concurrent is not None else None
    ranks = world if ours else 1
    total_ms = max_over_ranks(total_ms, ranks, device)
    ms_per_step = total_ms / args.steps
    raster_evals, voxel_evals, m2, m3 = step.eval_counts()
    evals_per_step = 2 * raster_evals + 2 * voxel_evals
    value = job_rate(evals_per_step, ranks, ms_per_step)

    e2e_ms, h2d, d2h = e2e_run(step, scene, args.steps, args.warmup, device)
    e2e_ms = max_over_ranks(e2e_ms, ranks, device)
    e2e_value = job_rate(evals_per_step, ranks, e2e_ms / args.steps)

    if stage_ms is None:
        stage_ms = ms_per_step
    api_ms = {k: v / stage_steps for k, v in api_stages.items()}
    api_ms["sum_of_stages"] = sum(api_ms.values())
    api_ms["outside_stages"] = stage_ms - api_ms["sum_of_stages"]

    peaks = measured_peaks()
    result = {
        "metric": WORKLOAD_TEXT[args.workload][0],
        "value": value,
        "unit": "evals/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "fit_steps_per_s": ranks * 1e3 / ms_per_step,
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
        "api_stages_ms_per_step": api_ms,
        "step_ms_distribution": ({"min": per_step[0], "median": statistics.median(per_step), "max": per_step[-1]}
                                 if per_step else None),
    }
    if not ours:
        launches = count_launches(step, scene)
        result.update({
            "impl": "reference",
            "gpu_launches": launches["all"] * args.steps,
            "launches_per_step": launches,
            "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "cpu_baseline": {
                "value": value, "unit": "evals/s", "cores": 1, "kind": "reference",
                "sample": "the reference's own package (explicit.py and its low-level wrapper, unmodified) on its "
                          "own CUDA kernels (compiled unmodified for sm_100a), driven by one host thread on the "
                          "same B200; the reference has no CPU implementation of these operators",
            },
        })
    else:
        result["gpu_launches"] = own_launches
        result["stages_ms_per_step"] = {k: v / stage_steps for k, v in stages.items()}
        if concurrent is not None:
            result["step_schedule"] = (
                "timed steps: the voxel half (voxelize_fwd, TV, voxelize_bwd) on a low-priority stream, issued "
                "first, and the raster half (rasterize_fwd with the loss epilogue, rasterize_bwd) on a "
                "high-priority stream; api_stages_ms_per_step, stages_ms_per_step and the rooflines come from "
                f"{stage_steps} steps run before them with both halves on one stream ({stage_ms:.3f} ms per step)")
            result["concurrent_stages"] = concurrent
        fp32_peak = fp32_peak_tflops(device)
        sfu_peak = sfu_peak_gops(device)
        result["rooflines"] = accumulate_rooflines(args.workload, stages, stage_steps, raster_evals, voxel_evals,
                                                   fp32_peak)
        result["roofline"] = dominant_roofline(args.workload, result["rooflines"], fp32_peak, sfu_peak,
                                               hbm_peak_gbs(peaks)[0])
        pack = pack_roofline(stages, stage_steps, int(scene.means.shape[0]), m3, *hbm_peak_gbs(peaks))
        if pack:
            result["rooflines"]["voxel_pack"] = pack
        if rank == 0 and not args.no_cpu_baseline and args.workload in ("ct", "small"):
            result["cpu_baseline"] = cpu_baseline(device, args.cpu_budget)
        if args.workload == "ct" and not args.no_mix and rank == 0:
            # Bounded runs of the multi-reconstruction forms, so the default line records them too.
            del step, scene, target, flush_buf
            torch.cuda.empty_cache()
            result["batched"] = bounded_mix(device, "batched")
            torch.cuda.empty_cache()
            result["served"] = bounded_mix(device, "serve")
    result["native_libs"] = mapped_native_libs()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))
    return 0


if __name__ == "__main__":
    sys.exit(main())
