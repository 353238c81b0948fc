"""Input validation for the explicit CT operators.

Mirrors the error contract of the reference's ``r2splat/_validation.py``
(``_shape`` :14-22, ``_scalar`` :25-32, ``_tensor`` :35-48, ``_constant``
:51-54, ``_vector`` :57-60, ``_primitives`` :63-86, ``_options`` :89-96): the
same exception types and messages are raised before any native call, because
callers and tests match on them.

The reference evaluates each value check (finiteness, ranges, camera
structure) with its own device reduction and host read. Here, inside
``deferred_value_checks()``, value checks are queued in the order they are
made and evaluated together by one kernel (``r2s_check_values``) and one host
read, when the block ends or when a host-side check raises; the first failing
check in call order raises, so the error a caller sees is the reference's.
"""

from __future__ import annotations

import contextlib
import ctypes
import math
import threading
from numbers import Integral, Real
from typing import Optional, Sequence, Union

import torch

Tensor = torch.Tensor
INT32_MAX = 2**31 - 1

# Check kinds of r2s_check_values (include/r2splat_b200.h).
FINITE, ZERO_ROW4, POSITIVE, NONNEGATIVE, FOCAL, PINHOLE, HOMOGENEOUS_ROW = range(7)
_ELEMENT_SIZE = {FINITE: 1, ZERO_ROW4: 4, POSITIVE: 1, NONNEGATIVE: 1, FOCAL: 9, PINHOLE: 9, HOMOGENEOUS_ROW: 16}


class _ValueCheck(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("count", ctypes.c_uint64), ("kind", ctypes.c_uint32),
                ("bit", ctypes.c_uint32)]


class _ValueChecks:
    """Value checks queued in call order: (tensor, kind, exception type, message)."""

    def __init__(self):
        self.items: list = []
        self._launched = None

    def launch(self) -> None:
        """Enqueues the queued checks: one kernel per (device, dtype, 32 checks) and an
        asynchronous copy of its flag word to pinned host memory, followed by an event."""
        items, self.items = self.items, []
        live = [(i, item) for i, item in enumerate(items) if item[0].numel() > 0]
        groups: dict = {}
        for index, item in live:
            groups.setdefault((item[0].device, item[0].dtype), []).append((index, item))
        from .cuda import _backend  # late import: the loader imports nothing from here

        words = []
        for (device, dtype), group in groups.items():
            for start in range(0, len(group), 32):
                chunk = group[start:start + 32]
                table = (_ValueCheck * len(chunk))()
                for bit, (_, (tensor, kind, _, _)) in enumerate(chunk):
                    table[bit] = _ValueCheck(tensor.data_ptr(), tensor.numel() // _ELEMENT_SIZE[kind], kind, bit)
                with torch.cuda.device(device):
                    stream = torch.cuda.current_stream(device)
                    flags = torch.empty(1, dtype=torch.int32, device=device)
                    _backend.call("r2s_check_values", 0 if dtype == torch.float32 else 1, table, len(chunk),
                                  flags.data_ptr(), stream.cuda_stream)
                    host = torch.empty(1, dtype=torch.int32, pin_memory=True)
                    host.copy_(flags, non_blocking=True)
                    done = torch.cuda.Event()
                    done.record(stream)
                words.append(([index for index, _ in chunk], host, done))
        self._launched = (items, words)

    def resolve(self):
        """Waits for the launched checks only (work queued after them keeps running);
        returns the first failing check's exception in call order, or None."""
        if self._launched is None:
            return None
        items, words = self._launched
        self._launched = None
        failed: set = set()
        for indices, host, done in words:
            done.synchronize()
            word = int(host[0])
            failed.update(index for bit, index in enumerate(indices) if word >> bit & 1)
        for index, (_, _, exc_type, message) in enumerate(items):
            if index in failed:
                return exc_type(message)
        return None

    def first_failure(self):
        """Evaluates the queued checks; returns the first failing one's exception, or None."""
        self.launch()
        return self.resolve()

    def check(self) -> None:
        """Raises the first failing launched check (see deferred_value_checks(pending=True))."""
        failure = self.resolve()
        if failure is not None:
            raise failure


_active = threading.local()


@contextlib.contextmanager
def deferred_value_checks(pending: bool = False):
    """Queue the value checks made inside the block and evaluate them with one host read.

    With ``pending=True`` the checks are only launched when the block ends; the
    caller enqueues its device work and then calls ``check()`` on the yielded
    object, which waits for the checks alone and raises the first failure, so
    the device does not idle on the read. Callers resolve before anything
    depends on the inputs being valid on the host (allocations sized from
    device counts, consuming a context).
    """
    checks = _ValueChecks()
    previous = getattr(_active, "checks", None)
    _active.checks = checks
    try:
        yield checks
    except BaseException:
        _active.checks = previous
        earlier = checks.first_failure()  # checks made before the failing host-side check
        if earlier is not None:
            raise earlier from None
        raise
    _active.checks = previous
    if pending:
        checks.launch()
        return
    failure = checks.first_failure()
    if failure is not None:
        raise failure


def _value_check(tensor: Tensor, kind: int, exc_type, message: str) -> None:
    """Fails with exc_type(message) if the check fails on any element (queued inside deferred_value_checks)."""
    checks = getattr(_active, "checks", None)
    if checks is not None:
        checks.items.append((tensor, kind, exc_type, message))
        return
    single = _ValueChecks()
    single.items.append((tensor, kind, exc_type, message))
    failure = single.first_failure()
    if failure is not None:
        raise failure


def _shape(name: str, value: Sequence[int], rank: int) -> tuple[int, ...]:
    if not isinstance(value, (tuple, list, torch.Size)) or len(value) != rank:
        raise ValueError(f"{name} must contain {rank} positive integers")
    for entry in value:
        if isinstance(entry, bool) or not isinstance(entry, Integral) or entry <= 0:
            raise ValueError(f"{name} must contain {rank} positive integers")
    result = tuple(int(entry) for entry in value)
    if math.prod(result) > INT32_MAX:
        raise ValueError(f"{name} exceeds the CUDA kernels' signed 32-bit indexing limit")
    return result


def _scalar(name: str, value: float, *, positive: bool = False) -> float:
    if isinstance(value, bool) or not isinstance(value, Real):
        raise TypeError(f"{name} must be a finite number")
    value = float(value)
    bad = value <= 0 if positive else value < 0
    if not math.isfinite(value) or bad:
        raise ValueError(f"{name} must be finite and {'positive' if positive else 'nonnegative'}")
    return value


def _tensor(name: str, value: Tensor, shape: tuple, reference: Optional[Tensor] = None) -> Tensor:
    if not isinstance(value, Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if value.ndim != len(shape) or any(want is not None and want != got for want, got in zip(shape, value.shape)):
        raise ValueError(f"{name} must have shape {shape}; got {tuple(value.shape)}")
    if value.dtype not in (torch.float32, torch.float64):
        raise TypeError(f"{name} must have dtype torch.float32 or torch.float64")
    if not value.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if reference is not None and (value.device != reference.device or value.dtype != reference.dtype):
        raise ValueError(f"{name} must have the same device and dtype as means")
    value = value.contiguous()
    _value_check(value, FINITE, ValueError, f"{name} must contain only finite values")
    return value


def _constant(name: str, value: Tensor) -> Tensor:
    if value.requires_grad:
        raise ValueError(f"gradients with respect to {name} are not supported")
    return value


def _vector(name: str, value: Union[Tensor, Sequence[float]], reference: Tensor) -> Tensor:
    if not isinstance(value, Tensor):
        value = torch.as_tensor(value, device=reference.device, dtype=reference.dtype)
    return _constant(name, _tensor(name, value, (3,), reference))


def _primitives(means, quats, scales, densities, beta, uncertainty):
    means = _tensor("means", means, (None, 3))
    n = means.shape[0]
    if n > INT32_MAX:
        raise ValueError("primitive count exceeds the CUDA kernels' signed 32-bit indexing limit")
    quats = _tensor("quats", quats, (n, 4), means)
    scales = _tensor("scales", scales, (n, 3), means)
    densities = _tensor("densities", densities, (n,), means)
    # Quaternions are normalised on the device; only all-zero rows are invalid.
    _value_check(quats, ZERO_ROW4, ValueError, "quats must have nonzero norm")
    _value_check(scales, POSITIVE, ValueError, "scales must be strictly positive physical lengths")
    _value_check(densities, NONNEGATIVE, ValueError, "densities must be nonnegative")
    if beta is not None:
        beta = _tensor("beta", beta, (n,), means)
        _value_check(beta, POSITIVE, ValueError, "beta must contain positive 3D exponents")
    if uncertainty is not None:
        uncertainty = _tensor("uncertainty", uncertainty, (n,), means)
        _value_check(uncertainty, NONNEGATIVE, ValueError, "uncertainty must be nonnegative relative variance")
    return means, quats, scales, densities, beta, uncertainty


def _options(beta, eps, radius_clip, detach_variance):
    if not isinstance(detach_variance, bool):
        raise TypeError("detach_variance must be a bool")
    eps = _scalar("eps", eps)
    if radius_clip is None:
        radius_clip = 3.0 if beta is None else 1.0
    radius_clip = _scalar("radius_clip", radius_clip, positive=True)
    return eps, radius_clip
