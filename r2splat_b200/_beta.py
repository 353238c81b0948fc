"""Line-integral factor of Beta primitives (host-side, float64).

A Beta density (1 - d^2)^gamma integrated along a ray has the Gaussian path
factor times B(1/2, gamma + 1) / sqrt(2 pi); the projected exponent is
gamma + 1/2. Behaviour follows the reference's ``r2splat/_beta.py``
(``beta_path_ratio`` :10-34, ``beta_path_log_grad`` :37-49): float64
evaluation with log-Gamma / digamma below gamma = 32 and an asymptotic series
in 1/z (z = gamma + 1) above, results cast back to the input dtype.

The series are the standard expansions
    log Gamma(z) - log Gamma(z + 1/2) = -log(z)/2 + 1/(8z) - 1/(192 z^3)
                                        + 1/(640 z^5) - 17/(14336 z^7) + ...
and its derivative in z. Both branches are evaluated on clamped inputs so
the inactive branch stays finite (no NaN through torch.where in autograd).
"""

from __future__ import annotations

import math

import torch

_SWITCH = 32.0


def beta_path_ratio(gamma: torch.Tensor) -> torch.Tensor:
    """B(1/2, gamma + 1) / sqrt(2 pi) for positive exponents gamma."""
    g = gamma.to(torch.float64)
    low = g.clamp_max(_SWITCH)
    exact = torch.lgamma(low + 1.0) - torch.lgamma(low + 1.5) - 0.5 * math.log(2.0)
    z = g.clamp_min(_SWITCH) + 1.0
    w = z.reciprocal()
    w2 = w * w
    series = w * (0.125 + w2 * (-1.0 / 192.0 + w2 * (1.0 / 640.0 - w2 * (17.0 / 14336.0))))
    tail = series - 0.5 * (math.log(2.0) + z.log())
    return torch.where(g < _SWITCH, exact, tail).exp().to(gamma.dtype)


def beta_path_log_grad(gamma: torch.Tensor) -> torch.Tensor:
    """d/dgamma of log B(1/2, gamma + 1)."""
    g = gamma.to(torch.float64)
    low = g.clamp_max(_SWITCH)
    exact = torch.special.digamma(low + 1.0) - torch.special.digamma(low + 1.5)
    w = (g.clamp_min(_SWITCH) + 1.0).reciprocal()
    w2 = w * w
    tail = w * (-0.5 + w * (-0.125 + w2 * (1.0 / 64.0 + w2 * (-1.0 / 128.0 + w2 * (17.0 / 2048.0)))))
    return torch.where(g < _SWITCH, exact, tail).to(gamma.dtype)


__all__ = ["beta_path_log_grad", "beta_path_ratio"]
