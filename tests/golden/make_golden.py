"""Generates the golden fixtures in tests/golden/ from the reference checkout.

Run where the reference checkout is readable, naming it by argument or by the
R2SPLAT_REFERENCE environment variable:
    python tests/golden/make_golden.py --reference <checkout>

Outputs (small, committed):
* dense_oracle.pt -- the reference's own float64 test oracle
  (tests/_reference.py: rasterize_reference / voxelize_reference) evaluated on
  seeded scenes of this repository's generator, with VJPs for fixed adjoints,
  over the Gaussian / Beta x plain / uncertainty / detached-variance matrix;
* beta_references.json -- the 160-digit Gamma/digamma reference values held by
  the reference's tests/test_beta_stability.py (REFERENCES);
* tile_bounds_3d.json -- the 3D tile-clipping cases of the reference's
  tests/test_tile_bounds.py (12 placements on a 3x2x4 grid of 4-voxel tiles);
* tv_reference.pt -- total variation value and gradient of a seeded [1,4,5,6]
  volume from the autograd edge-mean formula of tests/test_tv_loss.py.
"""

from __future__ import annotations

import argparse
import ast
import importlib.util
import json
import os
import sys
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def load_reference_oracle(reference: Path):
    spec = importlib.util.spec_from_file_location("reference_dense_oracle", reference / "tests" / "_reference.py")
    module = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(module)
    return module


def literal_assignment(path: Path, name: str):
    tree = ast.parse(path.read_text())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(getattr(t, "id", None) == name for t in node.targets):
            return ast.literal_eval(node.value)
    raise KeyError(name)


def _constant_expression(node):
    """Evaluates a literal, also allowing list(range(n)) as the test file writes it."""
    try:
        return ast.literal_eval(node)
    except ValueError:
        code = compile(ast.Expression(node), "<case>", "eval")
        return eval(code, {"__builtins__": {}}, {"list": list, "range": range})


def tile_bound_cases(path: Path):
    """Extracts the pytest.param(mean, radius, expected_ids, id=...) cases."""
    tree = ast.parse(path.read_text())
    cases = []
    for node in ast.walk(tree):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", None) == "param":
            values = [_constant_expression(a) for a in node.args]
            ident = next((ast.literal_eval(k.value) for k in node.keywords if k.arg == "id"), None)
            if len(values) == 3 and isinstance(values[0], tuple):
                cases.append({"mean": list(values[0]), "radius": values[1], "expected_ids": values[2], "id": ident})
    return cases


def scene_inputs(seed: int, n: int, beta: bool, uncertainty: bool):
    from r2splat_b200 import scenes

    means, quats, scales, densities, b, q = scenes.random_primitives(
        n, seed, 0.18, 0.25, beta_range=(0.8, 4.0) if beta else None, uncertainty_max=0.3 if uncertainty else None,
        dtype=torch.float64)
    means = means * 0.5
    viewmats, Ks = scenes.orbit_cameras(2, 2.5, 20.0, 20, 14, dtype=torch.float64)
    return dict(means=means, quats=quats, scales=scales, densities=densities, beta=b, uncertainty=q,
                viewmats=viewmats, Ks=Ks)


def dense_cases(oracle):
    cases = []
    names = ("means", "quats", "scales", "densities", "beta", "uncertainty")
    for idx, (beta, unc, detach) in enumerate([(False, False, False), (True, False, False), (False, True, False),
                                               (True, True, False), (False, True, True), (True, True, True)]):
        inputs = scene_inputs(100 + idx, 6, beta, unc)
        leaves = {k: v.clone().requires_grad_(True) for k, v in inputs.items()
                  if k in names and v is not None}
        options = dict(beta=leaves.get("beta"), uncertainty=leaves.get("uncertainty"), eps=0.01,
                       detach_variance=detach)
        prims = [leaves[k] for k in names[:4]]
        for op in ("rasterize", "voxelize"):
            if op == "rasterize":
                out = oracle.rasterize_reference(*prims, inputs["viewmats"], inputs["Ks"], (14, 20), **options)
            else:
                out = oracle.voxelize_reference(*prims, (5, 7, 9), volume_extent=(1.4, 1.6, 1.8),
                                                volume_center=(0.0, 0.05, -0.05), **options)
            outs = out if isinstance(out, tuple) else (out,)
            gen = torch.Generator().manual_seed(7 + idx)
            adjoints = [torch.randn(o.shape, generator=gen, dtype=torch.float64) for o in outs]
            loss = sum((o * a).sum() for o, a in zip(outs, adjoints))
            keys = [k for k in names if k in leaves]
            grads = torch.autograd.grad(loss, [leaves[k] for k in keys], allow_unused=True)
            cases.append({
                "op": op, "beta": beta, "uncertainty": unc, "detach": detach,
                "inputs": {k: v for k, v in inputs.items() if v is not None},
                "outputs": [o.detach() for o in outs], "adjoints": adjoints,
                "grads": {k: (torch.zeros_like(leaves[k]) if g is None else g.detach()) for k, g in zip(keys, grads)},
            })
    return cases


def tv_case():
    gen = torch.Generator().manual_seed(0)
    volume = torch.randn(1, 4, 5, 6, generator=gen, dtype=torch.float64).requires_grad_(True)
    diffs = [volume[:, 1:] - volume[:, :-1], volume[:, :, 1:] - volume[:, :, :-1],
             volume[:, :, :, 1:] - volume[:, :, :, :-1]]
    edges = sum(d.numel() for d in diffs)
    tv = sum(d.abs().sum() for d in diffs) / edges
    (grad,) = torch.autograd.grad(0.05 * tv, volume)
    return {"volume": volume.detach(), "lambda": 0.05, "tv": tv.detach(), "loss": 0.05 * tv.detach(), "grad": grad}


def main(argv=None) -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=os.environ.get("R2SPLAT_REFERENCE"),
                        help="reference checkout (default: $R2SPLAT_REFERENCE)")
    args = parser.parse_args(argv)
    if not args.reference:
        parser.error("give --reference or set R2SPLAT_REFERENCE")
    reference = Path(args.reference)
    oracle = load_reference_oracle(reference)
    torch.save(dense_cases(oracle), HERE / "dense_oracle.pt")
    refs = literal_assignment(reference / "tests" / "test_beta_stability.py", "REFERENCES")
    (HERE / "beta_references.json").write_text(json.dumps(
        {"source": "tests/test_beta_stability.py:11-22 (160-digit Gamma/digamma)",
         "columns": ["gamma", "ratio", "log_grad"], "rows": refs}, indent=1))
    cases = tile_bound_cases(reference / "tests" / "test_tile_bounds.py")
    (HERE / "tile_bounds_3d.json").write_text(json.dumps(
        {"source": "tests/test_tile_bounds.py:11-45", "grid": {"tile": 4, "tiles_x": 3, "tiles_y": 2, "tiles_z": 4},
         "cases": cases}, indent=1))
    torch.save(tv_case(), HERE / "tv_reference.pt")
    print("wrote", sorted(p.name for p in HERE.iterdir() if p.suffix in (".pt", ".json")))
    return 0


if __name__ == "__main__":
    sys.exit(main())
