"""The one-edit swap of the reference's low-level layer, run for real.

The reference resolves every low-level operator through
``importlib.import_module("r2splat.csrc")`` (``r2splat/cuda/_backend.py:29``).
Binding that name to ``r2splat_b200.cuda`` before the reference's package is
imported is the edit a maintainer makes; the reference's own ``explicit.py``
then runs unchanged on this library's kernels, operator by operator. This test
does that in a child process (the staged reference package, the same scenes)
and compares the results with the reference's package on its own kernels:
images and volumes bit for bit, gradients under the parity rule of _parity.py:
the 1e-5 / 1e-6 contract elementwise, and where an element is outside it (both
builds sum with atomics, in different orders), no farther from the float64 VJP
of the same fp32 forward, on the reference's kernels in float64, than the
reference build is. Each operator's own parity check against the reference
build is in test_low_level_reference_gpu.py.
"""

import subprocess
import sys
import textwrap
from pathlib import Path

import pytest
import torch

from _parity import assert_gradient_parity
from oracle import ref_ops
from r2splat_b200 import scenes

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_ops.package_available(), reason="staged reference package not present")]

ROOT = Path(__file__).resolve().parent.parent
FIELDS = ("means", "quats", "scales", "densities", "beta", "uncertainty")

CHILD = textwrap.dedent("""
    import sys, torch
    root, staged, backend, out_path = sys.argv[1:5]
    sys.path.insert(0, root)
    if backend == "b200":
        import r2splat_b200.cuda as module
    else:
        from oracle import ref_ops
        module = ref_ops.load()
    sys.modules["r2splat.csrc"] = module
    sys.path.insert(0, staged)
    import r2splat
    from r2splat_b200 import scenes
    dev = torch.device("cuda:0")
    out = {}
    for kind in ("gaussian", "beta"):
        if kind == "gaussian":
            sc = scenes.small_scene().to(dev)
            sc.uncertainty = None
        else:
            sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(dev)
        gen = torch.Generator().manual_seed(3)
        o, ctx = r2splat.rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                       uncertainty=sc.uncertainty)
        outs = o if isinstance(o, tuple) else (o,)
        adj = [torch.randn(t.shape, generator=gen).to(dev) for t in outs]
        g = r2splat.rasterize_bwd(ctx, *adj)
        vo, vctx = r2splat.voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                        uncertainty=sc.uncertainty)
        vouts = vo if isinstance(vo, tuple) else (vo,)
        vadj = [torch.randn(t.shape, generator=gen).to(dev) for t in vouts]
        vg = r2splat.voxelize_bwd(vctx, *vadj)
        out[kind] = {"outputs": [t.cpu() for t in outs], "voutputs": [t.cpu() for t in vouts],
                     "grads": [None if getattr(g, f) is None else getattr(g, f).cpu() for f in
                               ("means", "quats", "scales", "densities", "beta", "uncertainty")],
                     "vgrads": [None if getattr(vg, f) is None else getattr(vg, f).cpu() for f in
                                ("means", "quats", "scales", "densities", "beta", "uncertainty")]}
    torch.save(out, out_path)
""")


def _run(backend, tmp_path):
    out = tmp_path / f"{backend}.pt"
    proc = subprocess.run([sys.executable, "-c", CHILD, str(ROOT), str(ROOT / "oracle" / "_ref" / "py"), backend,
                           str(out)], capture_output=True, text=True, timeout=600)
    assert proc.returncode == 0, proc.stderr[-4000:]
    return torch.load(out, weights_only=False)


def _d(t):
    return None if t is None else t.double()


def _float64(saved):
    return {k: (v.double() if isinstance(v, torch.Tensor) and v.is_floating_point() else v) for k, v in saved.items()}


def _truths(kind, theirs):
    """The float64 raster and voxel VJPs of the child's fp32 forwards (the reference's kernels in float64), with
    the child's adjoints: the same scenes and the same generator sequence."""
    dev = torch.device("cuda:0")
    if kind == "gaussian":
        sc = scenes.small_scene().to(dev)
        sc.uncertainty = None
    else:
        sc = scenes.beta_scene(n=4096, cameras=8, side=64, focal=100.0, volume=32).to(dev)
    gen = torch.Generator().manual_seed(3)
    adj = [torch.randn(t.shape, generator=gen).to(dev) for t in theirs["outputs"]]
    _, saved = ref_ops.explicit_rasterize_fwd(*sc.primitives, sc.viewmats, sc.Ks, sc.image_size, beta=sc.beta,
                                              uncertainty=sc.uncertainty)
    raster = ref_ops.explicit_rasterize_bwd(_float64(saved), _d(sc.means), _d(sc.quats), _d(sc.scales), _d(sc.beta),
                                            _d(sc.uncertainty), *[_d(t) for t in adj], *([None] * (2 - len(adj))))
    vadj = [torch.randn(t.shape, generator=gen).to(dev) for t in theirs["voutputs"]]
    _, vsaved = ref_ops.explicit_voxelize_fwd(*sc.primitives, sc.volume_shape, volume_extent=(1, 1, 1), beta=sc.beta,
                                              uncertainty=sc.uncertainty)
    voxel = ref_ops.explicit_voxelize_bwd(_float64(vsaved), _d(sc.means), _d(sc.quats), _d(sc.scales),
                                          _d(sc.densities), _d(sc.beta), _d(sc.uncertainty), *[_d(t) for t in vadj],
                                          *([None] * (2 - len(vadj))))
    return {"grads": [None if t is None else t.cpu() for t in raster],
            "vgrads": [None if t is None else t.cpu() for t in voxel]}


def test_reference_explicit_runs_unchanged_on_this_library(tmp_path):
    mine = _run("b200", tmp_path)
    theirs = _run("reference", tmp_path)
    for kind in ("gaussian", "beta"):
        a, b = mine[kind], theirs[kind]
        for x, y in zip(a["outputs"] + a["voutputs"], b["outputs"] + b["voutputs"]):
            assert torch.equal(x, y), kind
        truth = _truths(kind, b)
        for key in ("grads", "vgrads"):
            for name, x, y, t in zip(FIELDS, a[key], b[key], truth[key]):
                if y is None:
                    assert x is None, (kind, key, name)
                    continue
                assert_gradient_parity(f"{kind} {key} {name}", x, y, t)
