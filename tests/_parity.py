"""Gradient parity against the reference build, shared by the GPU parity tests.

The contract is |ours - ref| <= 1e-6 + 1e-5 |ref| elementwise. Both builds sum
the same per-sample terms in fp32, in different orders (the reference with
atomics, this build record by record), so an element whose terms cancel can
differ by much more than 1e-5 of its value while both are equally close to the
exact sum. For the elements outside the contract the check therefore falls
back to the float64 VJP of the same fp32 forward, computed with the
reference's own kernels in float64 ("truth"): this build must be no farther
from it than the reference build is. "No farther" allows 25 % on three
statistics of the normalised error |x - truth| / (1e-6 + 1e-5 |truth|): the
norm-wise error (or, whichever is larger, the contract's relative 1e-5 applied
to the whole tensor), the count of elements above 1, and (for tensors of at
least 100,000 elements, where it is not just one of the few largest errors)
the 99.9th percentile. On
the 500k-primitive Beta scene with the variance branch (128 views at 768^2,
volume 384^3) these statistics of this build were 0.26 to 1.08 times the
reference build's.
"""

import torch


def contract_report(ours, ref):
    diff = (ours.double() - ref.double()).abs()
    bound = 1e-6 + 1e-5 * ref.double().abs()
    ratio = diff / bound
    return {"n": ours.numel(), "outside": int((ratio > 1).sum()),
            "max_excess": float(ratio.max()) if ours.numel() else 0.0,
            "relnorm": float(diff.norm() / ref.double().norm().clamp_min(1e-300))}


def truth_errors(x, truth):
    err = (x.double() - truth).abs() / (1e-6 + 1e-5 * truth.abs())
    flat = err.flatten()
    if flat.numel() > 8_000_000:
        flat = flat[torch.randperm(flat.numel(), device=flat.device)[:8_000_000]]
    return {"norm": float((x.double() - truth).norm()), "count": int((err > 1).sum()),
            "p999": float(torch.quantile(flat.float(), 0.999)) if flat.numel() else 0.0}


def assert_gradient_parity(name, ours, ref, truth=None, report=None):
    """The contract elementwise; elements outside it must be as accurate as the reference build's."""
    assert ours.shape == ref.shape and ours.dtype == ref.dtype, name
    stats = contract_report(ours, ref)
    if report is not None:
        report[name] = stats
    if stats["outside"] == 0:
        return stats
    assert truth is not None, f"{name}: {stats['outside']} elements outside 1e-5/1e-6, max excess {stats['max_excess']}"
    truth = truth.double()
    mine, theirs = truth_errors(ours, truth), truth_errors(ref, truth)
    stats.update(ours_vs_truth=mine, ref_vs_truth=theirs)
    norm_t = float(truth.norm())
    # Norm-wise: within 25 % of the reference's distance, or within the contract's relative 1e-5 of the
    # truth as a whole.
    assert mine["norm"] <= max(1.25 * theirs["norm"], 1e-5 * norm_t), (name, stats)
    assert mine["count"] <= 1.25 * theirs["count"] + 16, (name, stats)
    if ours.numel() >= 100_000:
        assert mine["p999"] <= 1.25 * theirs["p999"] + 0.05, (name, stats)
    return stats


def as_float64(value):
    """float64 copies of the floating tensors in value (a tensor, tuple, list or dict); others unchanged."""
    if isinstance(value, torch.Tensor):
        return value.double() if value.is_floating_point() else value
    if isinstance(value, dict):
        return {k: as_float64(v) for k, v in value.items()}
    if isinstance(value, (tuple, list)):
        return type(value)(as_float64(v) for v in value)
    return value
