"""Batched fit steps over many independent reconstructions, captured in one CUDA graph.

A ``FitScene`` owns one reconstruction on the device:
* its raw parameters: means, quats, log-scales, pre-softplus densities and log-beta, as in the
  reference's example fit loop (``examples/optimize.py``);
* their Adam moments and step counter;
* its cameras, target image and volume;
* every buffer one fit step touches, allocated once.

``FitScene.enqueue(stream)`` issues a whole fit step on ``stream`` with no host
synchronisation:
* raster forward (parameter transform, projection, capacity-bounded intersection lists,
  tile accumulation);
* the MSE image loss and its gradient ``2 (image - target) / numel``, written by
  the forward's tile kernel (fused epilogue);
* the record-parallel raster VJP and its chain rule;
* voxel forward, TV loss forward and backward in one pass, the voxel VJP and its chain rule;
* the fused activation-chain + Adam update.

The intersection counts stay on the device (``r2s_*_capacity`` entry points,
and the capacity-bounded form of the deterministic voxel VJP, whose slots are
the 3D intersections). When a count exceeds the scene's capacity, the step is
flagged and the update is skipped; ``BatchedFit`` then grows that capacity,
re-captures and the next replay redoes the step.

``BatchedFit`` captures the steps of all its scenes into one CUDA graph, each
scene on its own stream branch so that small scenes' kernels overlap, and
replays it: one launch per batched step. ``Autotuner`` picks each scene's
raster tile size (8, 16 or 32) and forward staging batch by timing eager steps,
caching the choice by scene shape.
"""

from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import _beta
from .cuda import _backend

Tensor = torch.Tensor
_DEFAULT_CAPACITY_SLACK = 1.3


def _p(t: Optional[Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _dt(t: Tensor) -> int:
    return 0 if t.dtype == torch.float32 else 1


def _ws(nbytes: int, device) -> Tensor:
    return torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=device)


@dataclass
class SceneConfig:
    """Geometry and optimisation settings of one reconstruction."""

    image_size: tuple
    volume_shape: tuple
    volume_extent: tuple = (1.0, 1.0, 1.0)
    volume_center: tuple = (0.0, 0.0, 0.0)
    tile: int = 16
    voxel_tile: int = 8
    stage_batch: int = 256
    lambda_tv: float = 0.05
    lr: float = 1e-3
    eps: float = 1e-8
    radius_clip: Optional[float] = None
    capacity_slack: float = _DEFAULT_CAPACITY_SLACK


class FitScene:
    """One reconstruction's parameters, Adam state and fit-step buffers on the device."""

    def __init__(self, means: Tensor, quats: Tensor, scales: Tensor, densities: Tensor, viewmats: Tensor,
                 Ks: Tensor, target: Tensor, config: SceneConfig, beta: Optional[Tensor] = None,
                 lean: bool = False):
        """``lean``: keep only what a fit continues from (parameters, activations, Adam state, cameras,
        target); the step buffers are not allocated and the scene is stepped through the explicit API
        (``serve.lean_step``), never by ``enqueue``."""
        self.cfg = config
        self.is_lean = bool(lean)
        self.device = means.device
        dev, dt = self.device, means.dtype
        n, c = means.shape[0], viewmats.shape[0]
        self.n, self.c = n, c
        self.height, self.width = config.image_size
        self.depth, self.vheight, self.vwidth = config.volume_shape
        self.radius_clip = config.radius_clip if config.radius_clip is not None else (3.0 if beta is None else 1.0)
        # Raw parameters (updated in place by the Adam step) and their activations.
        self.means = means.detach().clone().contiguous()
        self.quats = quats.detach().clone().contiguous()
        self.raw_scales = scales.detach().log().contiguous()
        d = densities.detach().to(torch.float64)
        self.raw_densities = torch.where(d > 20, d, torch.log(torch.expm1(d.clamp_min(1e-30)))).to(dt).contiguous()
        self.raw_beta = None if beta is None else beta.detach().log().contiguous()
        self.scales = self.raw_scales.exp()
        self.densities = torch.nn.functional.softplus(self.raw_densities)
        self.beta = None if self.raw_beta is None else self.raw_beta.exp()
        self.adam_m = torch.zeros((n, 12), dtype=dt, device=dev)
        self.adam_v = torch.zeros((n, 12), dtype=dt, device=dev)
        self.step_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.viewmats = viewmats.contiguous()
        self.Ks = Ks.contiguous()
        self.target = target.contiguous()
        self.extent = torch.tensor(config.volume_extent, dtype=dt, device=dev)
        self.center = torch.tensor(config.volume_center, dtype=dt, device=dev)
        self.overflow = torch.zeros(1, dtype=torch.int32, device=dev)
        self.loss = torch.zeros(1, dtype=dt, device=dev)
        self.ones = torch.ones(1, dtype=dt, device=dev)
        self._voxel_stream: Optional[torch.cuda.Stream] = None
        self.capacity_2d = 0
        self.capacity_3d = 0
        if self.is_lean:
            return
        self._allocate_fixed()
        self.set_capacity(*self.measure_counts())

    # ------------------------------------------------------------------ buffers
    def _allocate_fixed(self):
        dev, dt = self.device, self.means.dtype
        n, c, T = self.n, self.c, self.cfg.tile
        self.tx = (self.width + T - 1) // T
        self.ty = (self.height + T - 1) // T
        VT = self.cfg.voxel_tile
        self.vtx = (self.vwidth + VT - 1) // VT
        self.vty = (self.vheight + VT - 1) // VT
        self.vtz = (self.depth + VT - 1) // VT
        lib = _backend.library()
        self.covars = torch.empty((n, 6), dtype=dt, device=dev)
        self.max_scales = torch.empty((n,), dtype=dt, device=dev)
        self.records = torch.empty((c, n, 8), dtype=dt, device=dev)
        self.rects = torch.empty((c, n, 4), dtype=torch.int16, device=dev)
        self.counts = torch.empty((c, n), dtype=torch.int32, device=dev)
        self.cum = torch.empty((c * n,), dtype=torch.int64, device=dev)
        self.scan_ws = _ws(lib.r2s_isect_count_workspace(c * n), dev)
        self.offsets = torch.empty((c, self.ty, self.tx), dtype=torch.int32, device=dev)
        self.n_used = torch.zeros(1, dtype=torch.int64, device=dev)
        self.image = torch.empty((c, self.height, self.width), dtype=dt, device=dev)
        self.v_image = torch.empty_like(self.image)
        self.image_loss = torch.empty(1, dtype=dt, device=dev)
        self.image_loss_value = torch.empty(1, dtype=dt, device=dev)
        self.image_loss_ws = _ws(lib.r2s_raster_image_loss_workspace(c, self.tx, self.ty), dev)
        self.grads2d = torch.empty((c, n, 8), dtype=dt, device=dev)
        self.g_raster = [torch.empty((n, 3), dtype=dt, device=dev), torch.empty((n, 4), dtype=dt, device=dev),
                         torch.empty((n, 3), dtype=dt, device=dev), torch.empty((n,), dtype=dt, device=dev),
                         torch.empty((n,), dtype=dt, device=dev) if self.raw_beta is not None else None]
        # Voxel side.
        self.records3 = torch.empty((n, 16), dtype=dt, device=dev)
        self.means_v = torch.empty((n, 3), dtype=dt, device=dev)
        self.radii3 = torch.empty((n, 3), dtype=torch.int32, device=dev)
        self.counts3 = torch.empty((n,), dtype=torch.int32, device=dev)
        self.cum3 = torch.empty((n,), dtype=torch.int64, device=dev)
        self.scan3_ws = _ws(lib.r2s_isect_count_workspace(n), dev)
        self.offsets3 = torch.empty((self.vtz, self.vty, self.vtx), dtype=torch.int32, device=dev)
        self.n_used3 = torch.zeros(1, dtype=torch.int64, device=dev)
        self.volume = torch.empty((self.depth, self.vheight, self.vwidth), dtype=dt, device=dev)
        self.tv_ws = _ws(lib.r2s_volume_loss_workspace(self.volume.numel()), dev)
        self.tv_loss = torch.empty(1, dtype=dt, device=dev)
        self.tv_value = torch.empty(1, dtype=dt, device=dev)
        self.ones = torch.ones(1, dtype=dt, device=dev)
        self.g_volume = torch.empty_like(self.volume)
        self.grads3d = torch.empty((n, 16), dtype=dt, device=dev)
        self.g_voxel = [torch.empty((n, 3), dtype=dt, device=dev), torch.empty((n, 4), dtype=dt, device=dev),
                        torch.empty((n, 3), dtype=dt, device=dev), torch.empty((n,), dtype=dt, device=dev),
                        torch.empty((n,), dtype=dt, device=dev) if self.raw_beta is not None else None]

    def set_capacity(self, m2: int, m3: int):
        """(Re)allocates the intersection lists (and the voxel VJP's per-intersection slots) for m2 2D and
        m3 3D intersections plus slack."""
        dev = self.device
        lib = _backend.library()
        slack = self.cfg.capacity_slack
        self.capacity_2d = max(1024, int(math.ceil(m2 * slack)))
        self.capacity_3d = max(1024, int(math.ceil(m3 * slack)))
        self.slots3 = torch.empty((self.capacity_3d, 12), dtype=self.means.dtype, device=dev)
        self.isect_ids = torch.empty((self.capacity_2d,), dtype=torch.int64, device=dev)
        self.flatten_ids = torch.empty((self.capacity_2d,), dtype=torch.int32, device=dev)
        self.emit_ws = _ws(lib.r2s_isect_emit_workspace(self.capacity_2d, self.c * self.tx * self.ty), dev)
        self.isect3_ids = torch.empty((self.capacity_3d,), dtype=torch.int64, device=dev)
        self.flatten3_ids = torch.empty((self.capacity_3d,), dtype=torch.int32, device=dev)
        # Per-tile packed 3D records (list order, VJP slot in the padding) for the bulk-staged tile kernels.
        self.packed3 = torch.empty((self.capacity_3d, 16), dtype=self.means.dtype, device=dev)
        self.pack3_ws = _ws(lib.r2s_voxel_pack_workspace(self.n), dev)
        self.emit3_ws = _ws(lib.r2s_isect_emit_workspace(self.capacity_3d, self.vtx * self.vty * self.vtz), dev)

    def measure_counts(self) -> tuple[int, int]:
        """2D and 3D intersection counts of the current parameters (host read; used outside capture)."""
        stream = torch.cuda.current_stream(self.device).cuda_stream
        self._transform(stream)
        self._project(stream)
        self._project3(stream)
        torch.cuda.current_stream(self.device).synchronize()
        if not self.n:
            return 0, 0
        m2, m3 = torch.stack((self.cum[-1], self.cum3[-1])).tolist()
        return int(m2), int(m3)

    def needs_capacity(self) -> tuple[int, int]:
        """(m2, m3) of the current parameters; call after a flagged overflow."""
        return self.measure_counts()

    # ------------------------------------------------------------------ kernels
    def _transform(self, stream):
        """Covariances from the activated quaternions and scales (read by both halves of the step)."""
        d = _dt(self.means)
        _backend.call("r2s_parameter_transform_fwd", d, _p(self.quats), _p(self.scales), _p(self.covars),
                      _p(self.max_scales), self.n, stream)

    def _project(self, stream):
        d = _dt(self.means)
        self.ratio = _beta.beta_path_ratio(self.beta) if self.beta is not None else None
        _backend.call("r2s_raster_project", d, _p(self.means), _p(self.covars), _p(self.densities), _p(self.beta),
                      _p(self.ratio), _p(self.viewmats), _p(self.Ks), self.c, self.n, self.width, self.height,
                      float(self.cfg.eps), float(self.cfg.eps), float(self.radius_clip), self.cfg.tile, self.tx,
                      self.ty, _p(self.records), _p(self.rects), _p(self.counts), stream)
        _backend.call("r2s_scan_tile_counts", _p(self.counts), self.c * self.n, _p(self.cum), _p(self.scan_ws),
                      self.scan_ws.numel(), stream)

    def _project3(self, stream):
        d = _dt(self.means)
        _backend.call("r2s_voxel_project", d, _p(self.means), _p(self.covars), _p(self.densities), _p(self.beta),
                      None, _p(self.extent), _p(self.center), self.n, self.vwidth, self.vheight, self.depth,
                      float(self.cfg.eps), float(self.radius_clip), self.cfg.voxel_tile, self.vtx, self.vty, self.vtz,
                      _p(self.records3), _p(self.means_v), _p(self.radii3), _p(self.counts3), stream)
        _backend.call("r2s_scan_tile_counts", _p(self.counts3), self.n, _p(self.cum3), _p(self.scan3_ws),
                      self.scan3_ws.numel(), stream)

    def enqueue(self, stream: torch.cuda.Stream):
        """Issues one complete fit step on `stream` (capturable: no host synchronisation).

        The raster half runs on `stream`; the voxel half (projection, lists, forward, TV, VJP,
        chain rule) forks onto a stream of the scene's own and joins back before the update, so
        the two halves' kernels overlap on the device (and in a captured graph they are two
        branches). Both read the covariances computed before the fork; neither reads what the other
        writes, and both only raise the shared overflow flag.
        """
        s = stream.cuda_stream
        d = _dt(self.means)
        beta_flag = int(self.beta is not None)
        if self._voxel_stream is None:
            self._voxel_stream = torch.cuda.Stream(device=self.device)
        vstream = self._voxel_stream
        with torch.cuda.stream(stream):
            self.overflow.zero_()
            self._transform(s)
        vstream.wait_stream(stream)
        self._enqueue_voxel_half(vstream, d, beta_flag)
        with torch.cuda.stream(stream):
            # Raster forward, loss gradient, VJP.
            self._project(s)
            _backend.call("r2s_raster_emit_capacity", _p(self.rects), self.c, self.n, self.tx, self.ty, _p(self.cum),
                          self.capacity_2d, _p(self.n_used), _p(self.overflow), _p(self.isect_ids),
                          _p(self.flatten_ids), _p(self.offsets), _p(self.emit_ws), self.emit_ws.numel(), s)
            # Tile forward with the MSE image loss and its gradient in the epilogue.
            _backend.call("r2s_raster_render_image_loss", d, _p(self.records), None, beta_flag, _p(self.offsets),
                          _p(self.flatten_ids), 0, _p(self.n_used), self.c, self.n, self.width, self.height,
                          self.cfg.tile, self.tx, self.ty, self.cfg.stage_batch, _p(self.target), 0, 1.0,
                          _p(self.image), None, _p(self.v_image), _p(self.image_loss), _p(self.image_loss_value),
                          _p(self.image_loss_ws), self.image_loss_ws.numel(), s)
            _backend.call("r2s_raster_record_bwd", d, _p(self.records), _p(self.rects), None, beta_flag, 0,
                          _p(self.v_image), None, self.c, self.n, self.width, self.height, self.cfg.tile,
                          _p(self.grads2d), None, None, s)
            log_grad = _beta.beta_path_log_grad(self.beta) if self.beta is not None else None
            g = self.g_raster
            _backend.call("r2s_raster_chain_bwd", d, _p(self.means), _p(self.quats), _p(self.scales),
                          _p(self.covars), _p(self.beta), _p(self.ratio), _p(log_grad), _p(self.viewmats),
                          _p(self.Ks), self.c, self.n, self.width, self.height, float(self.cfg.eps),
                          float(self.cfg.eps), _p(self.grads2d), _p(g[0]), _p(g[1]), _p(g[2]), _p(g[3]), _p(g[4]), s)
            stream.wait_stream(vstream)
            # Loss (image MSE + lambda TV), then the update unless this step overflowed.
            torch.add(self.image_loss, self.tv_loss, out=self.loss)
            grads_a = (ctypes.c_void_p * 5)(*[None if t is None else t.data_ptr() for t in self.g_raster])
            grads_b = (ctypes.c_void_p * 5)(*[None if t is None else t.data_ptr() for t in self.g_voxel])
            self._grad_tables = (grads_a, grads_b)  # kept alive for the captured call's duration
            _backend.call("r2s_adam_activation_step", d, self.n, _p(self.means), _p(self.quats),
                          _p(self.raw_scales), _p(self.raw_densities), _p(self.raw_beta), _p(self.scales),
                          _p(self.densities), _p(self.beta), _p(self.adam_m), _p(self.adam_v), grads_a, grads_b,
                          float(self.cfg.lr), 0.9, 0.999, 1e-8, _p(self.step_count), _p(self.overflow), s)

    def _enqueue_voxel_half(self, stream: torch.cuda.Stream, d: int, beta_flag: int):
        """Voxel forward, TV, VJP and chain rule of one fit step on `stream`."""
        s = stream.cuda_stream
        with torch.cuda.stream(stream):
            self._project3(s)
            _backend.call("r2s_voxel_emit_capacity", d, _p(self.means_v), _p(self.radii3), self.n,
                          self.cfg.voxel_tile, self.vtx, self.vty, self.vtz, _p(self.cum3), self.capacity_3d,
                          _p(self.n_used3), _p(self.overflow), _p(self.isect3_ids), _p(self.flatten3_ids),
                          _p(self.offsets3), _p(self.emit3_ws), self.emit3_ws.numel(), s)
            _backend.call("r2s_voxel_pack_tile_records", d, _p(self.records3), _p(self.offsets3),
                          _p(self.flatten3_ids), _p(self.radii3), _p(self.cum3), self.n, self.capacity_3d,
                          _p(self.n_used3), self.cfg.voxel_tile, self.vtx, self.vty, self.vtz, self.capacity_3d,
                          _p(self.packed3), _p(self.pack3_ws), self.pack3_ws.numel(), s)
            _backend.call("r2s_voxel_render_packed", d, _p(self.packed3), beta_flag, _p(self.offsets3), 0,
                          _p(self.n_used3), self.vwidth, self.vheight, self.depth, self.cfg.voxel_tile, self.vtx,
                          self.vty, self.vtz, _p(self.volume), None, s)
            # TV forward and backward in one pass (the TV term enters the loss with weight one).
            _backend.call("r2s_volume_loss_fwd_bwd", d, _p(self.volume), _p(self.ones), 1, self.depth, self.vheight,
                          self.vwidth, float(self.cfg.lambda_tv), _p(self.tv_loss), _p(self.tv_value), None,
                          _p(self.g_volume), _p(self.tv_ws), self.tv_ws.numel(), s)
            # Deterministic tile VJP: one slot per 3D intersection, summed per primitive in a fixed order.
            _backend.call("r2s_voxel_render_bwd_packed", d, _p(self.packed3), beta_flag, 1, _p(self.offsets3), 0,
                          _p(self.n_used3), _p(self.cum3), _p(self.g_volume), None, self.n, self.vwidth,
                          self.vheight, self.depth, self.cfg.voxel_tile, self.vtx, self.vty, self.vtz,
                          _p(self.slots3), self.capacity_3d, _p(self.grads3d), s)
            v = self.g_voxel
            _backend.call("r2s_voxel_chain_bwd", d, _p(self.means), _p(self.quats), _p(self.scales), _p(self.covars),
                          _p(self.extent), _p(self.center), self.n, self.vwidth, self.vheight, self.depth,
                          float(self.cfg.eps), _p(self.grads3d), _p(v[0]), _p(v[1]), _p(v[2]), _p(v[3]), _p(v[4]),
                          None, s)

    def step(self):
        """One eager fit step on the current stream (grows the capacity and repeats on overflow)."""
        stream = torch.cuda.current_stream(self.device)
        while True:
            self.enqueue(stream)
            if int(self.overflow.item()) == 0:
                return
            self.set_capacity(*self.needs_capacity())

    # ------------------------------------------------------------------ snapshot / restore
    STATE_KEYS = ("means", "quats", "raw_scales", "raw_densities", "raw_beta", "scales", "densities", "beta",
                  "adam_m", "adam_v", "step_count")

    def state_dict(self) -> dict:
        """Host copies of everything a fit continues from: the raw parameters, their activations (as the
        update kernel wrote them, so a restore needs no recomputation that could round differently), the
        Adam moments and the step counter."""
        torch.cuda.current_stream(self.device).synchronize()
        return {k: None if getattr(self, k) is None else getattr(self, k).detach().cpu().clone()
                for k in self.STATE_KEYS}

    def load_state_dict(self, state: dict):
        """Copies a ``state_dict`` back in place (the buffers keep their addresses, so a captured graph of
        this scene stays valid). The scene must have the same primitive count and kind."""
        for k in self.STATE_KEYS:
            dst, src = getattr(self, k), state[k]
            if (dst is None) != (src is None):
                raise ValueError(f"state {k!r} does not match this scene (Gaussian vs Beta)")
            if dst is None:
                continue
            if tuple(dst.shape) != tuple(src.shape) or dst.dtype != src.dtype:
                raise ValueError(f"state {k!r} has shape {tuple(src.shape)} {src.dtype}, this scene "
                                 f"{tuple(dst.shape)} {dst.dtype}")
            dst.copy_(src, non_blocking=False)


class BatchedFit:
    """Fit steps of many FitScenes as one CUDA graph: one replay per batched step."""

    def __init__(self, scenes: Sequence[FitScene]):
        self.scenes = list(scenes)
        self.device = self.scenes[0].device
        self.streams = [torch.cuda.Stream(device=self.device) for _ in self.scenes]
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        self.flags = torch.zeros(len(self.scenes), dtype=torch.int32, device=self.device)
        self.recaptures = 0

    def capture(self, warm: bool = True):
        """Captures one batched step. warm: first run one eager step per scene (a real step), so that
        kernel attributes and lazy module loading happen outside capture."""
        if warm:
            for scene in self.scenes:
                scene.step()
        torch.cuda.synchronize(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            origin = torch.cuda.current_stream(self.device)
            for s in self.streams:
                s.wait_stream(origin)
            for scene, s in zip(self.scenes, self.streams):
                scene.enqueue(s)
            for s in self.streams:
                origin.wait_stream(s)
            torch.stack([scene.overflow[0] for scene in self.scenes], out=self.flags)
        self.graph = graph

    def step(self, check: bool = True):
        """Replays one batched fit step; with check, re-plans and redoes overflowed scenes."""
        if self.graph is None:
            self.capture()
        self.graph.replay()
        if not check:
            return
        flags = self.flags.tolist()
        if any(flags):
            for scene, flag in zip(self.scenes, flags):
                if flag:
                    scene.set_capacity(*scene.needs_capacity())
                    scene.step()  # the skipped step, now with room
            self.recaptures += 1
            self.graph = None
            self.capture(warm=False)

    def losses(self) -> list[float]:
        return [float(scene.loss.item()) for scene in self.scenes]


class Autotuner:
    """Picks (raster tile size, forward staging batch) per scene shape by timing eager fit steps."""

    TILES = (8, 16, 32)
    BATCHES = (64, 128, 256)

    def __init__(self, steps: int = 2):
        self.steps = steps
        self.cache: dict = {}

    @staticmethod
    def key(n: int, cameras: int, image_size: tuple, kind: str) -> tuple:
        return (int(round(math.log2(max(n, 1)))), cameras, tuple(image_size), kind)

    def choose(self, make_scene, n: int, cameras: int, image_size: tuple, kind: str) -> tuple[int, int]:
        """make_scene(tile, stage_batch) -> FitScene. Returns the fastest (tile, stage_batch)."""
        k = self.key(n, cameras, image_size, kind)
        if k in self.cache:
            return self.cache[k]
        best, best_ms = (16, 256), float("inf")
        for tile in self.TILES:
            for batch in self.BATCHES:
                if tile == 8 and batch > 64:
                    continue  # an 8x8 tile has 64 pixels: the staging batch is capped at the thread count
                scene = make_scene(tile, batch)
                scene.step()
                torch.cuda.synchronize()
                start = time.perf_counter()
                for _ in range(self.steps):
                    scene.step()
                torch.cuda.synchronize()
                ms = (time.perf_counter() - start) * 1e3 / self.steps
                if ms < best_ms:
                    best, best_ms = (tile, batch), ms
                del scene
        self.cache[k] = best
        return best


def make_synthetic_scene(n: int, cameras: int, side: int, volume: int, *, beta: bool = False, seed: int = 0,
                         tile: int = 16, stage_batch: int = 256, lr: float = 1e-3, device="cuda",
                         dtype=torch.float32, lean: bool = False) -> FitScene:
    """A seeded reconstruction in the CT benchmark's distributions.

    Primitives: scales exp(N(log 0.01, 0.4)). Cameras: an orbit of radius 3 with focal length
    1.17 x side. The target image is rendered from means perturbed by N(0, 0.005).
    """
    from . import explicit, scenes

    means, quats, scales, densities, b, _ = scenes.random_primitives(
        n, seed, 0.01, 0.4, beta_range=(0.5, 4.0) if beta else None, dtype=dtype)
    viewmats, Ks = scenes.orbit_cameras(cameras, 3.0, 1.171875 * side, side, side, dtype=dtype)
    to = (lambda t: None if t is None else t.to(device))
    means, quats, scales, densities, b, viewmats, Ks = map(to, (means, quats, scales, densities, b, viewmats, Ks))
    shifted = scenes.perturbed_means(means, seed=seed + 2)
    target, _ = explicit.rasterize_fwd(shifted, quats, scales, densities, viewmats, Ks, (side, side), beta=b)
    config = SceneConfig(image_size=(side, side), volume_shape=(volume, volume, volume), tile=tile,
                         stage_batch=stage_batch, lr=lr)
    return FitScene(means, quats, scales, densities, viewmats, Ks, target, config, beta=b, lean=lean)


__all__ = ["Autotuner", "BatchedFit", "FitScene", "SceneConfig", "make_synthetic_scene"]
