"""The drop-in explicit operators: forward passes that hand back a one-shot VJP context.

Public surface and error contract of the reference's ``r2splat/explicit.py``:
``rasterize_fwd`` (:102-188), ``rasterize_bwd`` (:191-242), ``voxelize_fwd``
(:245-311), ``voxelize_bwd`` (:314-351) and ``ParameterGradients`` (:25-34).
No autograd graph is built. A forward returns its output detached plus a
context; the matching backward accepts that context exactly once, refuses it
if any tensor it captured was written in place since, and returns the
gradients as a ``ParameterGradients`` without touching ``.grad``. Cameras,
volume extent and centre are constants; activations and loss derivatives are
the caller's.

Device work runs through the fused sm_100a pipelines of ``_fused``. Both
``backward_mode`` values are accepted and run the same VJP (in the reference
they select two kernels that differ only in float summation order).
"""

from __future__ import annotations

import contextlib
from dataclasses import dataclass
from typing import Optional, Sequence, Union

import torch

from . import _fused
from ._validation import (FOCAL, HOMOGENEOUS_ROW, PINHOLE, POSITIVE, _constant, _options, _primitives, _shape,
                          _tensor, _value_check, _vector, deferred_value_checks)

Tensor = torch.Tensor
Output = Union[Tensor, tuple[Tensor, Tensor]]
_PRIMITIVE_NAMES = ("means", "quats", "scales", "densities", "beta", "uncertainty")
# Launch geometry bounds of the reference's kernels, kept as input limits of the contract.
_GRID_LIMIT = 65535
_INDEX_LIMIT = 2**31 - 1


@dataclass
class ParameterGradients:
    """Gradients with respect to the physical inputs of a forward call.

    ``beta`` and ``uncertainty`` are None when the forward had no such input.
    """

    means: Tensor
    quats: Tensor
    scales: Tensor
    densities: Tensor
    beta: Optional[Tensor] = None
    uncertainty: Optional[Tensor] = None


class _Context:
    """What one forward call leaves for its backward, usable once.

    ``versions`` holds ``(name, tensor, version)`` for every distinct tensor
    the forward read or produced for the backward; ``open`` compares them
    again, so an in-place write in between is reported instead of silently
    giving wrong gradients.
    """

    __slots__ = ("kind", "shape", "primitives", "buffers", "versions", "eps", "backward_mode",
                 "detach_variance", "used")

    def __init__(self, kind, shape, primitives, buffers, versions, eps, backward_mode, detach_variance):
        self.kind, self.shape, self.eps = kind, shape, eps
        self.primitives, self.buffers, self.versions = primitives, buffers, versions
        self.backward_mode, self.detach_variance = backward_mode, detach_variance
        self.used = False

    @classmethod
    def capture(cls, kind, shape, primitives, buffers, originals, eps, backward_mode, detach_variance):
        """A context that watches the caller's originals, the validated primitives and the saved tensors."""
        named = [*originals, *zip(_PRIMITIVE_NAMES, primitives), *buffers.items()]
        versions, ids = [], set()
        for name, value in named:
            if not isinstance(value, Tensor) or id(value) in ids:
                continue
            ids.add(id(value))
            try:
                versions.append((name, value, value._version))
            except RuntimeError as error:  # inference tensors carry no version counter
                raise ValueError("explicit contexts require tensors with version counters") from error
        return cls(kind, shape, primitives, buffers, tuple(versions), eps, backward_mode, detach_variance)

    def open(self, kind):
        """Checks that this is an unused, unmodified context of a ``kind`` forward."""
        if self.kind != kind:
            raise TypeError(f"expected a context returned by {kind}_fwd")
        if self.used:
            raise RuntimeError("this context has already been consumed by backward")
        stale = next((name for name, value, version in self.versions if value._version != version), None)
        if stale is not None:
            raise RuntimeError(f"saved input {stale} was modified in-place after forward")

    def close(self, gradients):
        """Marks the context used, drops every reference it holds and passes ``gradients`` through."""
        self.used = True
        self.primitives, self.versions = (), ()
        self.buffers.clear()
        return gradients

    def adjoint(self, name, value):
        """``value`` checked against the forward output's shape, device and dtype (None passes through)."""
        return None if value is None else _tensor(name, value, self.shape, self.primitives[0])

    def zero_gradients(self):
        return ParameterGradients(*(None if p is None else torch.zeros_like(p) for p in self.primitives))


def _open_context(context, kind):
    if not isinstance(context, _Context):
        raise TypeError(f"expected a context returned by {kind}_fwd")
    context.open(kind)


@contextlib.contextmanager
def _resolving(checks):
    """Resolves pending input checks after the block's device work is enqueued.

    A failing check is raised in preference to an error of the block itself.
    Checks already resolved inside the block (before a host read) are not
    evaluated again.
    """
    try:
        yield
    except BaseException:
        failure = checks.resolve()
        if failure is not None:
            raise failure from None
        raise
    checks.check()


def _backward_mode(value):
    mode = str(value).lower()
    if mode in ("pixel", "primitive"):
        return mode
    raise ValueError("backward_mode must be 'pixel' or 'primitive'")


def release_intersection_lists(context) -> None:
    """Frees a forward context's intersection lists before its backward runs.

    Not part of the reference's surface: a memory-bounded caller (the serving
    loop's recompute-in-backward mode) calls it between ``rasterize_fwd`` /
    ``voxelize_fwd`` and the matching backward. Neither VJP reads the lists:
    the raster VJP walks each record's tile rectangle and the voxel VJP then
    walks each primitive's tile box. The gradients are unchanged up to the
    voxel VJP's summation order.
    """
    if not isinstance(context, _Context) or context.used:
        raise RuntimeError("expected an unconsumed explicit context")
    state = context.buffers.get("state")
    if state is None:
        return
    dropped = {id(t) for t in _fused.release_lists(state)}
    for key in ("offsets", "isect_ids", "flatten_ids"):
        context.buffers.pop(key, None)
    context.versions = tuple(entry for entry in context.versions if id(entry[1]) not in dropped)


def _context(kind, shape, primitives, buffers, originals, eps, mode, detach_variance):
    return _Context.capture(kind, shape, primitives, buffers, originals, eps, mode, detach_variance)


@torch.no_grad()
def rasterize_fwd(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    densities: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    image_size: Sequence[int],
    *,
    beta: Optional[Tensor] = None,
    uncertainty: Optional[Tensor] = None,
    eps: float = 1.0e-8,
    radius_clip: Optional[float] = None,
    detach_variance: bool = False,
    backward_mode: str = "primitive",
) -> tuple[Output, _Context]:
    """Line-integral images of the primitives for every camera, plus the context for ``rasterize_bwd``.

    ``viewmats [C,4,4]`` (world to camera) and the pinhole intrinsics ``Ks
    [C,3,3]`` are constants. The output is ``[C,height,width]``, or the pair
    ``(image, variance)`` when ``uncertainty`` is given; it never carries an
    autograd graph, and the inputs need not require grad.
    """
    return _rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, beta, uncertainty, eps,
                          radius_clip, detach_variance, backward_mode, None)


def rasterize_fwd_with_loss(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    densities: Tensor,
    viewmats: Tensor,
    Ks: Tensor,
    image_size: Sequence[int],
    target: Tensor,
    *,
    loss: str = "mse",
    loss_weight: float = 1.0,
    beta: Optional[Tensor] = None,
    uncertainty: Optional[Tensor] = None,
    eps: float = 1.0e-8,
    radius_clip: Optional[float] = None,
    detach_variance: bool = False,
    backward_mode: str = "primitive",
) -> tuple[Output, _Context, Tensor, Tensor, Tensor]:
    """``rasterize_fwd`` with the mean image loss against ``target`` fused into the tile kernel.

    No reference counterpart: the reference's fit loop (examples/optimize.py)
    computes the image loss and its gradient with separate passes after the
    forward; its L1 form is ``image_loss_l1_fwd/bwd`` (Loss.cpp:12-113). Here
    the tile kernel's epilogue writes them while the image is in registers.

    ``target`` is ``[C,height,width]`` with the primitives' device and dtype.
    ``loss`` is "mse" (``weight * mean((image - target)^2)``, gradient
    ``(image - target) * (2 weight / numel)``) or "l1" (``weight * mean|image -
    target|``, gradient ``weight * sign(image - target) / numel``, the
    reference's L1 backward with an upstream gradient of one). The loss is on
    the image only; with ``uncertainty`` the variance is returned as usual.

    Returns ``(output, context, v_image, loss, loss_value)``: ``v_image`` is
    the adjoint to pass to ``rasterize_bwd``; ``loss`` is the weighted mean
    (0-dim) and ``loss_value`` the unweighted one, both summed in fp64 in a
    fixed order.
    """
    if loss not in _fused.IMAGE_LOSS_KINDS:
        raise ValueError('loss must be "mse" or "l1"')
    weight = float(loss_weight)
    if not (weight == weight and abs(weight) != float("inf")):
        raise ValueError("loss_weight must be finite")
    return _rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, beta, uncertainty, eps,
                          radius_clip, detach_variance, backward_mode, (target, loss, weight))


def _rasterize_fwd(means, quats, scales, densities, viewmats, Ks, image_size, beta, uncertainty, eps, radius_clip,
                   detach_variance, backward_mode, image_loss):
    originals = list(zip(
        ("means", "quats", "scales", "densities", "viewmats", "Ks", "beta", "uncertainty"),
        (means, quats, scales, densities, viewmats, Ks, beta, uncertainty),
    ))
    with deferred_value_checks(pending=True) as checks:
        height, width = _shape("image_size", image_size, 2)
        primitives = _primitives(means, quats, scales, densities, beta, uncertainty)
        means, quats, scales, densities, beta, uncertainty = primitives
        eps, radius_clip = _options(beta, eps, radius_clip, detach_variance)
        mode = _backward_mode(backward_mode)
        # requires_grad must be judged on the caller's tensors: _tensor may hand back a
        # contiguous copy, and under no_grad that copy no longer requires grad.
        for name, value in (("viewmats", viewmats), ("Ks", Ks)):
            if isinstance(value, Tensor):
                _constant(name, value)
        viewmats = _constant("viewmats", _tensor("viewmats", viewmats, (None, 4, 4), means))
        cameras = viewmats.shape[0]
        if cameras == 0:
            raise ValueError("viewmats must contain at least one camera")
        largest_index = cameras * max(height * width, means.shape[0])
        if largest_index > _INDEX_LIMIT or cameras > _GRID_LIMIT:
            raise ValueError("camera batch exceeds CUDA indexing or grid limits")
        if max(height, width) > _fused.RASTER_TILE * _GRID_LIMIT:
            raise ValueError("image_size exceeds CUDA grid limits")
        Ks = _constant("Ks", _tensor("Ks", Ks, (cameras, 3, 3), means))
        _value_check(Ks, FOCAL, ValueError, "Ks must have positive fx and fy")
        _value_check(Ks, PINHOLE, ValueError, "Ks must be pinhole intrinsics with zero skew and last row [0, 0, 1]")
        _value_check(viewmats, HOMOGENEOUS_ROW, ValueError, "viewmats must have homogeneous last row [0, 0, 0, 1]")
        if image_loss is not None:
            target = _constant("target", _tensor("target", image_loss[0], (cameras, height, width), means))
            image_loss = (target,) + tuple(image_loss[1:])
    shape = (cameras, height, width)
    buffers = {"viewmats": viewmats, "Ks": Ks}
    loss_out = None
    if means.shape[0] == 0:
        checks.check()
        image = means.new_zeros(shape)
        output = image if uncertainty is None else (image, image.clone())
        if image_loss is not None:
            # No primitives, no intersections: every tile list is empty.
            tile = _fused.RASTER_TILE
            offsets = torch.zeros((cameras * ((height + tile - 1) // tile) * ((width + tile - 1) // tile),),
                                  dtype=torch.int32, device=means.device)
            with torch.cuda.device(means.device):
                loss_out = _fused.render_image_loss(None, None, False, offsets, None, 0, 1, width, height, tile,
                                                    image_loss[0], image_loss[1], image_loss[2], image, None,
                                                    means.device)
    else:
        with _resolving(checks), torch.cuda.device(means.device):
            # The input checks resolve just before the intersection count is read.
            result = _fused.raster_forward(means, quats, scales, densities, viewmats, Ks, width, height, beta,
                                           uncertainty, eps, radius_clip, image_loss=image_loss,
                                           before_count=checks.check)
        output, state = result[0], result[1]
        if image_loss is not None:
            loss_out = result[2]
        buffers.update(state=state, covars=state.covars, records=state.records, offsets=state.offsets,
                       isect_ids=state.isect_ids, flatten_ids=state.flatten_ids, ratio=state.ratio)
    context = _context("rasterize", shape, primitives, buffers, originals, eps, mode, detach_variance)
    if image_loss is None:
        return output, context
    return (output, context) + tuple(loss_out)


@torch.no_grad()
def rasterize_bwd(context: _Context, v_image: Optional[Tensor], v_variance: Optional[Tensor] = None
                  ) -> ParameterGradients:
    """Gradients of ``<output, adjoint>`` with respect to the primitives, from a ``rasterize_fwd`` context.

    Each adjoint has the shape, device and dtype of the output it belongs to;
    None stands for a zero adjoint (so a loss on the variance alone passes
    ``v_image=None``). The context is used up, and the forward's inputs must
    not have been modified in place since the forward.
    """
    _open_context(context, "rasterize")
    means, quats, scales, densities, beta, uncertainty = context.primitives
    if v_variance is not None and uncertainty is None:
        raise ValueError("v_variance requires uncertainty in the forward call")
    with deferred_value_checks(pending=True) as checks:
        v_image = context.adjoint("v_image", v_image)
        v_variance = context.adjoint("v_variance", v_variance)
    if means.shape[0] == 0 or (v_image is None and v_variance is None):
        checks.check()
        return context.close(context.zero_gradients())
    b = context.buffers
    # The VJP is enqueued before the adjoint checks resolve; on a failure its
    # result is dropped and the context stays unconsumed.
    with _resolving(checks), torch.cuda.device(means.device):
        grads = _fused.raster_backward(b["state"], means, quats, scales, densities, beta, uncertainty,
                                       b["viewmats"], b["Ks"], context.eps, v_image, v_variance,
                                       context.detach_variance)
    return context.close(ParameterGradients(*grads))


@torch.no_grad()
def voxelize_fwd(
    means: Tensor,
    quats: Tensor,
    scales: Tensor,
    densities: Tensor,
    volume_shape: Sequence[int],
    *,
    volume_extent: Union[Tensor, Sequence[float]],
    volume_center: Union[Tensor, Sequence[float]] = (0.0, 0.0, 0.0),
    beta: Optional[Tensor] = None,
    uncertainty: Optional[Tensor] = None,
    eps: float = 1.0e-8,
    radius_clip: Optional[float] = None,
    detach_variance: bool = False,
    backward_mode: str = "primitive",
) -> tuple[Output, _Context]:
    """Densities of the primitives sampled at voxel centres, plus the context for ``voxelize_bwd``.

    ``volume_shape`` and the output are ``[depth,height,width]``; the
    physical ``volume_extent`` and ``volume_center`` are given in x, y, z
    order. With ``uncertainty`` the output is ``(volume, variance)``.
    """
    originals = list(zip(
        ("means", "quats", "scales", "densities", "volume_extent", "volume_center", "beta", "uncertainty"),
        (means, quats, scales, densities, volume_extent, volume_center, beta, uncertainty),
    ))
    with deferred_value_checks(pending=True) as checks:
        depth, height, width = _shape("volume_shape", volume_shape, 3)
        if max(height, width) > _fused.VOXEL_TILE * _GRID_LIMIT:
            raise ValueError("volume_shape exceeds CUDA grid limits")
        primitives = _primitives(means, quats, scales, densities, beta, uncertainty)
        means, quats, scales, densities, beta, uncertainty = primitives
        eps, radius_clip = _options(beta, eps, radius_clip, detach_variance)
        mode = _backward_mode(backward_mode)
        for name, value in (("volume_extent", volume_extent), ("volume_center", volume_center)):
            if isinstance(value, Tensor):
                _constant(name, value)
        extent = _vector("volume_extent", volume_extent, means)
        center = _vector("volume_center", volume_center, means)
        _value_check(extent, POSITIVE, ValueError, "volume_extent must contain positive physical lengths")
    shape = (depth, height, width)
    buffers = {"extent": extent, "center": center}
    if means.shape[0] == 0:
        checks.check()
        volume = means.new_zeros(shape)
        output = volume if uncertainty is None else (volume, volume.clone())
    else:
        with _resolving(checks), torch.cuda.device(means.device):
            output, state = _fused.voxel_forward(means, quats, scales, densities, shape, extent, center, beta,
                                                 uncertainty, eps, radius_clip, before_count=checks.check)
        buffers.update(state=state, covars=state.covars, records=state.records, offsets=state.offsets,
                       isect_ids=state.isect_ids, flatten_ids=state.flatten_ids)
    context = _context("voxelize", shape, primitives, buffers, originals, eps, mode, detach_variance)
    return output, context


@torch.no_grad()
def voxelize_bwd(context: _Context, v_volume: Optional[Tensor], v_variance: Optional[Tensor] = None
                 ) -> ParameterGradients:
    """Gradients of ``<volume, adjoint>`` with respect to the primitives, from a ``voxelize_fwd`` context.

    Adjoint rules as for ``rasterize_bwd``; no input's ``.grad`` is written.
    """
    _open_context(context, "voxelize")
    means, quats, scales, densities, beta, uncertainty = context.primitives
    if v_variance is not None and uncertainty is None:
        raise ValueError("v_variance requires uncertainty in the forward call")
    with deferred_value_checks(pending=True) as checks:
        v_volume = context.adjoint("v_volume", v_volume)
        v_variance = context.adjoint("v_variance", v_variance)
    if means.shape[0] == 0 or (v_volume is None and v_variance is None):
        checks.check()
        return context.close(context.zero_gradients())
    b = context.buffers
    with _resolving(checks), torch.cuda.device(means.device):
        grads = _fused.voxel_backward(b["state"], means, quats, scales, beta, uncertainty, b["extent"],
                                      b["center"], context.eps, v_volume, v_variance, context.detach_variance)
    return context.close(ParameterGradients(*grads))


# rasterize_fwd_with_loss is an extension outside the reference's surface: it is
# reached as r2splat_b200.explicit.rasterize_fwd_with_loss and not re-exported.
__all__ = ["ParameterGradients", "rasterize_fwd", "rasterize_bwd", "voxelize_fwd", "voxelize_bwd"]
