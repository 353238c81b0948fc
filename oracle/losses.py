"""TV and image-L1 oracle (numpy, float64 accumulation) -- TEST INFRASTRUCTURE ONLY.

TV follows ``VolumeLossFwd.cu:39-82`` + ``Loss.cpp:115-152`` (mean absolute
forward difference over all edges of a [B,D,H,W] volume, times lambda) and
``VolumeLossBwd.cu:46-115`` + ``Loss.cpp:154-188`` (sign sums times g/edges,
times lambda). L1 follows ``ImageLossFwd.cu:19-31`` / ``ImageLossBwd.cu:14-30``.
"""

from __future__ import annotations

import numpy as np


def tv_forward(volume, lambda_tv):
    v = np.asarray(volume, dtype=np.float64)
    diffs = [np.diff(v, axis=a) for a in (1, 2, 3)]
    edges = max(sum(d.size for d in diffs), 1)
    tv_map = np.zeros_like(v)
    tv_map[:, :-1] += np.abs(diffs[0])
    tv_map[:, :, :-1] += np.abs(diffs[1])
    tv_map[:, :, :, :-1] += np.abs(diffs[2])
    tv = tv_map.sum() / edges
    return lambda_tv * tv, tv, tv_map


def tv_backward(volume, grad_output, lambda_tv):
    v = np.asarray(volume, dtype=np.float64)
    diffs = [np.diff(v, axis=a) for a in (1, 2, 3)]
    edges = max(sum(d.size for d in diffs), 1)
    g = np.zeros_like(v)
    s = [np.sign(d) for d in diffs]
    g[:, :-1] -= s[0]
    g[:, 1:] += s[0]
    g[:, :, :-1] -= s[1]
    g[:, :, 1:] += s[1]
    g[:, :, :, :-1] -= s[2]
    g[:, :, :, 1:] += s[2]
    return g * (float(np.asarray(grad_output).reshape(-1)[0]) / edges) * lambda_tv


def l1_forward(prediction, target, lambda_l1):
    m = np.abs(np.asarray(prediction, np.float64) - np.asarray(target, np.float64))
    l1 = m.mean() if m.size else 0.0
    return lambda_l1 * l1, l1, m


def l1_backward(prediction, target, grad_output, lambda_l1):
    d = np.asarray(prediction, np.float64) - np.asarray(target, np.float64)
    return float(np.asarray(grad_output).reshape(-1)[0]) * lambda_l1 * np.sign(d) / max(d.size, 1)


__all__ = ["l1_backward", "l1_forward", "tv_backward", "tv_forward"]
