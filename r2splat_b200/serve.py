"""Continuous-batching fit-step server over many resident reconstructions.

Requests name a reconstruction and ask for one fit step of it. The server
keeps every admitted reconstruction's parameters and Adam moments resident on
the device, and runs requests as follows:

* Admission is by an HBM budget. Lean steps run one at a time, and the
  largest transient peak of a lean step (measured by its first step at
  admission) is held back from the budget. A reconstruction whose full
  fit-step footprint (all buffers of a ``FitScene`` plus its captured graph)
  fits the rest is kept *graphed*: one CUDA-graph replay per step. The
  graph's private memory is only known after capture; if it tips the total
  over the budget, the graph is dropped and the reconstruction kept lean. One
  that does not fit is kept *lean*: parameters, Adam moments, cameras and target
  resident, every other buffer allocated for the step and released after it.
  A lean step runs the explicit API (which rebuilds the intersection lists each
  step) plus the same fused activation + Adam update. A reconstruction that
  does not fit even lean waits until memory frees up.
* Scheduling is continuous. A scheduler thread of control launches each
  arrived request as soon as its reconstruction has no step in flight and one
  of ``slots`` CUDA streams is free, so requests that arrive while others run
  are started immediately and their kernels overlap on the device. A graphed
  step is one replay. A lean step reads intersection counts back to the host
  while it runs, so it runs on a worker thread of its own: the scheduler keeps
  launching graphed steps on the other streams meanwhile, and a large lean
  reconstruction does not hold up the small ones. Completion is detected with
  CUDA events; latency is arrival to completion.
* A graphed step whose intersection lists outgrow their capacity skips its
  update and raises the scene's overflow flag; each replay copies that flag
  to pinned host memory ahead of its completion event. On completion the
  server grows the capacity, redoes the step eagerly and captures the graph
  again, so every completed request is one applied update.
* Requests for a reconstruction that is still waiting for memory are dropped
  and counted (``ServeStats.rejected``); a key that was never offered raises
  ``KeyError`` before anything runs.

``snapshot(key)`` / ``restore(key, snapshot)`` copy a reconstruction's
parameters, activations, Adam moments and step counter to host memory and
back; a restored reconstruction continues bit for bit as the original would.

``serve()`` replays a list of (arrival time, reconstruction) requests against
the wall clock and reports fit-steps/s with p50/p99 latency. ``serve_serially``
runs the same requests one at a time through the plain explicit API: the
baseline the served form is compared with.
"""

from __future__ import annotations

import ctypes
import heapq
import time
from collections import deque
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field
from typing import Callable, Optional

import torch

from . import batched, explicit
from .cuda import _backend
from .cuda import _wrapper as low

Tensor = torch.Tensor


@dataclass
class Reconstruction:
    key: object
    scene: batched.FitScene
    graphed: bool
    graph: Optional[torch.cuda.CUDAGraph] = None
    busy: bool = False
    steps: int = 0
    footprint: int = 0
    overflow_host: Optional[Tensor] = None  # pinned copy of the scene's overflow flag after each replay


@dataclass
class ServeStats:
    completed: int
    wall_s: float
    latencies_ms: list = field(default_factory=list)
    lean: int = 0
    graphed: int = 0
    waited_for_memory: int = 0
    rejected: int = 0
    regrown: int = 0
    lean_latencies_ms: list = field(default_factory=list)

    @property
    def steps_per_s(self) -> float:
        return self.completed / self.wall_s if self.wall_s > 0 else 0.0

    def percentile(self, q: float, values: Optional[list] = None) -> float:
        values = sorted(self.latencies_ms if values is None else values)
        if not values:
            return float("nan")
        index = min(len(values) - 1, max(0, int(round(q / 100.0 * (len(values) - 1)))))
        return values[index]

    def summary(self) -> dict:
        out = {"completed": self.completed, "wall_s": self.wall_s, "fit_steps_per_s": self.steps_per_s,
               "p50_ms": self.percentile(50), "p99_ms": self.percentile(99), "graphed": self.graphed,
               "lean": self.lean, "waited_for_memory": self.waited_for_memory, "rejected": self.rejected,
               "regrown": self.regrown}
        if self.lean_latencies_ms:
            lean = self.lean_latencies_ms
            other = sorted(self.latencies_ms)
            for x in lean:
                other.remove(x)
            out.update(lean_requests=len(lean), lean_p50_ms=self.percentile(50, lean),
                       lean_p99_ms=self.percentile(99, lean), graphed_p50_ms=self.percentile(50, other),
                       graphed_p99_ms=self.percentile(99, other))
        return out


def lean_step(scene: batched.FitScene, recompute: bool = False):
    """One fit step through the explicit API with transient buffers, then the fused update.

    ``recompute``: free each forward's intersection lists before its backward (the raster VJP never reads
    them; the voxel VJP then walks the primitives' tile boxes), so the lists of the two passes are never
    resident at the same time as the backward's buffers.
    """
    cfg = scene.cfg
    _, ctx, v_image, image_loss, _ = explicit.rasterize_fwd_with_loss(
        scene.means, scene.quats, scene.scales, scene.densities, scene.viewmats, scene.Ks, cfg.image_size,
        scene.target, loss="mse", beta=scene.beta, eps=cfg.eps, radius_clip=cfg.radius_clip)
    if recompute:
        explicit.release_intersection_lists(ctx)
    g = explicit.rasterize_bwd(ctx, v_image)
    volume, vctx = explicit.voxelize_fwd(scene.means, scene.quats, scene.scales, scene.densities, cfg.volume_shape,
                                         volume_extent=cfg.volume_extent, volume_center=cfg.volume_center,
                                         beta=scene.beta, eps=cfg.eps, radius_clip=cfg.radius_clip)
    if recompute:
        explicit.release_intersection_lists(vctx)
    tv, _, g_vol = low.volume_loss_fwd_bwd(volume.unsqueeze(0), scene.ones, cfg.lambda_tv)
    gv = explicit.voxelize_bwd(vctx, g_vol[0])
    torch.add(image_loss.reshape(1), tv.reshape(1), out=scene.loss)
    ga = (ctypes.c_void_p * 5)(*[None if t is None else t.data_ptr() for t in (g.means, g.quats, g.scales,
                                                                               g.densities, g.beta)])
    gb = (ctypes.c_void_p * 5)(*[None if t is None else t.data_ptr() for t in (gv.means, gv.quats, gv.scales,
                                                                               gv.densities, gv.beta)])
    _backend.call("r2s_adam_activation_step", 0 if scene.means.dtype == torch.float32 else 1, scene.n,
                  ctypes.c_void_p(scene.means.data_ptr()), ctypes.c_void_p(scene.quats.data_ptr()),
                  ctypes.c_void_p(scene.raw_scales.data_ptr()), ctypes.c_void_p(scene.raw_densities.data_ptr()),
                  None if scene.raw_beta is None else ctypes.c_void_p(scene.raw_beta.data_ptr()),
                  ctypes.c_void_p(scene.scales.data_ptr()), ctypes.c_void_p(scene.densities.data_ptr()),
                  None if scene.beta is None else ctypes.c_void_p(scene.beta.data_ptr()),
                  ctypes.c_void_p(scene.adam_m.data_ptr()), ctypes.c_void_p(scene.adam_v.data_ptr()), ga, gb,
                  float(cfg.lr), 0.9, 0.999, 1e-8, ctypes.c_void_p(scene.step_count.data_ptr()), None,
                  torch.cuda.current_stream().cuda_stream)


class FitServer:
    """Admits reconstructions against an HBM budget and serves fit-step requests continuously."""

    def __init__(self, budget_bytes: int, slots: int = 8, device="cuda", lean_recompute: bool = False,
                 lean_reserve_bytes: int = 0):
        """``lean_recompute``: lean reconstructions free each forward's intersection lists before the
        backward (``lean_step(recompute=True)``), for budgets that large reconstructions press against.
        ``lean_reserve_bytes``: memory held back for lean steps from the start (it grows to the largest
        transient peak measured at a lean admission)."""
        self.device = torch.device(device)
        self.lean_recompute = bool(lean_recompute)
        self.budget = int(budget_bytes)
        self.used = 0
        # Peak transient memory of one lean step (the largest measured at admission). Lean steps run one at
        # a time, so this much of the budget is held back from resident reconstructions.
        self.lean_reserve = int(lean_reserve_bytes)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(slots)]
        self.recons: dict = {}
        self.waiting: deque = deque()  # (key, factory) not yet admitted
        # Lean steps run here, one at a time, so their host reads do not stall the scheduler.
        self._lean_worker = ThreadPoolExecutor(max_workers=1, thread_name_prefix="r2s-lean-step")
        self._lean_future: Optional[Future] = None

    # ----------------------------------------------------------- admission
    def admit(self, key, factory: Callable[[], batched.FitScene]) -> bool:
        """Creates and admits a reconstruction; returns False (queued) when memory is short."""
        torch.cuda.synchronize(self.device)
        before = torch.cuda.memory_allocated(self.device)
        scene = factory()
        torch.cuda.synchronize(self.device)
        full = torch.cuda.memory_allocated(self.device) - before
        recon, warm_steps = None, 0
        if not scene.is_lean and self.used + full + self.lean_reserve <= self.budget:
            recon = Reconstruction(key, scene, graphed=True, footprint=full)
            self._capture(recon)
            if self.used + recon.footprint + self.lean_reserve > self.budget:
                # The graph's private pool tipped it over: keep it lean instead (its warm-up step stays applied).
                warm_steps, recon.graph, recon = recon.steps, None, None
                torch.cuda.synchronize(self.device)
        if recon is None:
            # Lean: release every fit-step buffer; keep parameters, moments, cameras, target.
            self._make_lean(scene)
            torch.cuda.synchronize(self.device)
            lean = torch.cuda.memory_allocated(self.device) - before
            transient = 0
            fits = self.used + lean + self.lean_reserve <= self.budget
            if fits and warm_steps == 0:
                # One real step measures the lean step's transient peak (and warms the scene up, as a
                # graphed admission's first step does).
                torch.cuda.reset_peak_memory_stats(self.device)
                base = torch.cuda.memory_allocated(self.device)
                try:
                    lean_step(scene, recompute=self.lean_recompute)
                    torch.cuda.synchronize(self.device)
                    transient = torch.cuda.max_memory_allocated(self.device) - base
                    warm_steps = 1
                except torch.cuda.OutOfMemoryError:
                    fits = False
            fits = fits and self.used + lean + max(self.lean_reserve, transient) <= self.budget
            if not fits:
                del scene
                torch.cuda.empty_cache()
                self.waiting.append((key, factory))
                return False
            self.lean_reserve = max(self.lean_reserve, transient)
            recon = Reconstruction(key, scene, graphed=False, footprint=lean, steps=warm_steps)
        self.used += recon.footprint
        self.recons[key] = recon
        return True

    @staticmethod
    def _make_lean(scene: batched.FitScene):
        keep = {"means", "quats", "raw_scales", "raw_densities", "raw_beta", "scales", "densities", "beta",
                "adam_m", "adam_v", "step_count", "viewmats", "Ks", "target", "extent", "center", "loss", "ones",
                "cfg", "device", "n", "c", "height", "width", "depth", "vheight", "vwidth", "radius_clip"}
        for name in list(vars(scene)):
            if name not in keep and isinstance(getattr(scene, name), (torch.Tensor, list)):
                setattr(scene, name, None)
        scene.is_lean = True

    def _capture(self, recon: Reconstruction, warm: bool = True):
        """Captures the reconstruction's fit step; ``warm`` first runs one real eager step outside capture."""
        scene = recon.scene
        if warm:
            scene.step()
            recon.steps += 1
        if recon.overflow_host is None:
            recon.overflow_host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        torch.cuda.synchronize(self.device)
        before = torch.cuda.memory_allocated(self.device)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            scene.enqueue(torch.cuda.current_stream(self.device))
        torch.cuda.synchronize(self.device)
        recon.footprint += torch.cuda.memory_allocated(self.device) - before
        recon.graph = graph

    # ----------------------------------------------------------- snapshot / restore
    def snapshot(self, key) -> dict:
        """Host copy of a resident reconstruction's parameters, activations, Adam moments and step counter.

        Waits for the reconstruction's work in flight on the device; call it between ``serve()`` runs.
        """
        recon = self.recons[key]
        torch.cuda.synchronize(self.device)
        return {"steps": recon.steps, "state": recon.scene.state_dict()}

    def restore(self, key, snapshot: dict):
        """Puts a snapshot back into an admitted reconstruction of the same shape; its captured graph
        (if any) stays valid, since the state is copied into the same device buffers."""
        recon = self.recons[key]
        torch.cuda.synchronize(self.device)
        recon.scene.load_state_dict(snapshot["state"])
        recon.steps = snapshot["steps"]

    def evict(self, key):
        recon = self.recons.pop(key)
        self.used -= recon.footprint
        del recon
        torch.cuda.synchronize(self.device)
        while self.waiting:
            k, factory = self.waiting[0]
            if not self.admit(k, factory):
                self.waiting.pop()  # admit() queued it again at the back; keep its place at the front
                self.waiting.appendleft((k, factory))
                break
            self.waiting.popleft()

    # ----------------------------------------------------------- serving
    def _launch(self, recon: Reconstruction, stream: torch.cuda.Stream):
        """Starts one step on ``stream``; returns an object whose ``query()`` is True once it is done."""
        if recon.graphed:
            with torch.cuda.stream(stream):
                recon.graph.replay()
                recon.overflow_host.copy_(recon.scene.overflow, non_blocking=True)
                done = torch.cuda.Event()
                done.record(stream)
            return done
        recompute = self.lean_recompute

        def run():
            with torch.cuda.device(self.device), torch.cuda.stream(stream):
                lean_step(recon.scene, recompute=recompute)
                done = torch.cuda.Event()
                done.record(stream)
            return done

        self._lean_future = self._lean_worker.submit(run)
        return _LeanStep(self._lean_future)

    def _wait_lean(self):
        """Waits for the lean step on the worker thread, if any (re-raising its error)."""
        if self._lean_future is not None:
            self._lean_future.result().synchronize()

    def close(self):
        """Waits for a lean step in flight and stops the worker thread."""
        try:
            self._wait_lean()
        finally:
            self._lean_worker.shutdown(wait=True)

    def _finish(self, recon: Reconstruction, stats: ServeStats):
        """Completion of a step: a graphed step that overflowed is redone with room, then re-captured."""
        if not recon.graphed or int(recon.overflow_host[0]) == 0:
            return
        scene = recon.scene
        # Capturing while the worker thread launches a lean step would put its work into the graph.
        self._wait_lean()
        torch.cuda.synchronize(self.device)
        before = torch.cuda.memory_allocated(self.device)
        recon.graph = None
        scene.set_capacity(*scene.needs_capacity())
        scene.step()  # the skipped update, now with room (it grows again if it must)
        self._capture(recon, warm=False)
        torch.cuda.synchronize(self.device)
        grown = torch.cuda.memory_allocated(self.device) - before
        recon.footprint += grown
        self.used += grown
        stats.regrown += 1

    def serve(self, requests: list, poll_s: float = 2e-5) -> ServeStats:
        """requests: [(arrival_s, key)] relative to the call. Runs every request of an admitted reconstruction.

        Requests for reconstructions still waiting for memory are dropped and
        counted in ``rejected``; a key the server has never been offered raises
        KeyError before anything runs.
        """
        waiting = {key for key, _ in self.waiting}
        unknown = sorted({repr(key) for _, key in requests if key not in self.recons and key not in waiting})
        if unknown:
            raise KeyError(f"requests name reconstructions that were never admitted: {', '.join(unknown)}")
        pending: dict = {key: deque() for key in self.recons}
        rejected = sum(1 for _, key in requests if key not in self.recons)
        arrivals = deque(sorted((r for r in requests if r[1] in self.recons), key=lambda r: r[0]))
        free = list(range(len(self.streams)))
        in_flight: list = []  # (event, slot, key, arrival)
        ready: list = []  # heap of (arrival, seq, key)
        stats = ServeStats(0, 0.0)
        stats.graphed = sum(r.graphed for r in self.recons.values())
        stats.lean = len(self.recons) - stats.graphed
        stats.waited_for_memory = len(self.waiting)
        stats.rejected = rejected
        seq = 0
        lean_in_flight = 0
        start = time.perf_counter()
        while arrivals or in_flight or ready or any(pending.values()):
            now = time.perf_counter() - start
            while arrivals and arrivals[0][0] <= now:
                t, key = arrivals.popleft()
                pending[key].append(t)
                if len(pending[key]) == 1 and not self.recons[key].busy:
                    heapq.heappush(ready, (t, seq, key))
                    seq += 1
            progressed = False
            still = []
            for event, slot, key, t in in_flight:
                if event.query():
                    recon = self.recons[key]
                    lean_in_flight -= int(not recon.graphed)
                    self._finish(recon, stats)
                    stats.completed += 1
                    latency = (time.perf_counter() - start - t) * 1e3
                    stats.latencies_ms.append(latency)
                    if not recon.graphed:
                        stats.lean_latencies_ms.append(latency)
                    recon.busy = False
                    recon.steps += 1
                    free.append(slot)
                    if pending[key]:
                        heapq.heappush(ready, (pending[key][0], seq, key))
                        seq += 1
                    progressed = True
                else:
                    still.append((event, slot, key, t))
            in_flight = still
            deferred = []
            while free and ready:
                item = heapq.heappop(ready)
                t, _, key = item
                recon = self.recons[key]
                if not recon.graphed and lean_in_flight:
                    deferred.append(item)  # lean steps run one at a time (their transient is reserved once)
                    continue
                pending[key].popleft()
                recon.busy = True
                lean_in_flight += int(not recon.graphed)
                slot = free.pop()
                in_flight.append((self._launch(recon, self.streams[slot]), slot, key, t))
                progressed = True
            for item in deferred:
                heapq.heappush(ready, item)
            if not progressed:
                time.sleep(poll_s)
        stats.wall_s = time.perf_counter() - start
        self._wait_lean()
        return stats


class _LeanStep:
    """A lean step running on the worker thread: done once the thread has launched it and its event fired."""

    def __init__(self, future: Future):
        self.future = future

    def query(self) -> bool:
        if not self.future.done():
            return False
        return self.future.result().query()  # re-raises an error of the step


def serve_serially(recons: dict, requests: list) -> ServeStats:
    """The baseline: each request's fit step through the plain explicit API, one at a time, in arrival order."""
    stats = ServeStats(0, 0.0)
    start = time.perf_counter()
    for t, key in sorted(requests, key=lambda r: r[0]):
        now = time.perf_counter() - start
        if t > now:
            time.sleep(t - now)
        lean_step(recons[key])
        torch.cuda.synchronize()
        stats.completed += 1
        stats.latencies_ms.append((time.perf_counter() - start - t) * 1e3)
    stats.wall_s = time.perf_counter() - start
    return stats


def poisson_requests(keys: list, rate_per_s: float, count: int, seed: int = 0) -> list:
    """`count` requests over `keys` (uniformly) with exponential inter-arrival times."""
    gen = torch.Generator().manual_seed(seed)
    gaps = torch.empty(count, dtype=torch.float64).exponential_(rate_per_s, generator=gen)
    times = torch.cumsum(gaps, 0).tolist()
    picks = torch.randint(len(keys), (count,), generator=gen).tolist()
    return [(t, keys[i]) for t, i in zip(times, picks)]


__all__ = ["FitServer", "ServeStats", "lean_step", "poisson_requests", "serve_serially"]
