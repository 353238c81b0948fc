"""Build recipe for the reference CUDA extension used as a parity checker.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module.

Two steps, both writing only under ``oracle/_ref/`` (git-ignored; it travels
with the working tree to the GPU host):

1. Compiles the reference's own low-level operator sources (``r2splat/cuda/csrc``
   of MedAPT-group/R2Splat, the files listed by its ``setup.py:17-22``)
   unmodified, from where they lie, with the reference's nvcc flags
   (``setup.py:29-34``: ``-O3 --use_fast_math -std=c++17
   --expt-relaxed-constexpr``) plus an explicit ``sm_100a`` target. The product
   is a torch extension module named ``r2splat_ref_csrc`` in ``oracle/_ref/``;
   intermediate objects go to ``oracle/_ref/build/``. It exposes the
   reference's 40 pybind names (``ext.cpp:8-183``).
2. Stages the reference's pure-Python package (``r2splat/**/*.py``: the public
   ``explicit.py`` surface, ``_validation.py``, ``_beta.py`` and the
   ``cuda`` loader/wrapper) into ``oracle/_ref/py/r2splat``, as a
   ``pip install --target`` of the package would place it. ``oracle.ref_ops``
   imports it with ``r2splat.csrc`` bound to the module of step 1, so the
   reference bench arm and the parity tests run the reference's own Python
   code on the reference's own kernels.

The reference checkout is given by ``--reference PATH`` or the
``R2SPLAT_REFERENCE`` environment variable; there is no default location.

Usage (needs the reference checkout, nvcc and ninja; no GPU):
    R2SPLAT_REFERENCE=<checkout> python oracle/build_ref.py [--jobs N] [--package-only]
"""

from __future__ import annotations

import argparse
import glob
import os
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
PACKAGE_OUT = OUT / "py"
MODULE = "r2splat_ref_csrc"
REFERENCE_ENV = "R2SPLAT_REFERENCE"


def reference_root(path: str | None = None) -> Path | None:
    """The reference checkout named by ``path`` or by $R2SPLAT_REFERENCE, if any."""
    value = path or os.environ.get(REFERENCE_ENV)
    return Path(value) if value else None


def built_module_path() -> Path | None:
    hits = sorted(OUT.glob(MODULE + "*.so"))
    return hits[0] if hits else None


def stage_package(reference: str | Path) -> Path:
    """Copies the reference's Python sources (no csrc) into ``oracle/_ref/py/r2splat``."""
    src = Path(reference) / "r2splat"
    if not (src / "__init__.py").is_file():
        raise FileNotFoundError(f"reference package not found under {src}")
    dst = PACKAGE_OUT / "r2splat"
    if dst.exists():
        shutil.rmtree(dst)
    for path in sorted(src.rglob("*.py")):
        target = dst / path.relative_to(src)
        target.parent.mkdir(parents=True, exist_ok=True)
        shutil.copy2(path, target)
    return dst


def build(reference: str | Path, jobs: int | None = None, verbose: bool = True) -> Path:
    src = Path(reference) / "r2splat" / "cuda" / "csrc"
    inc = Path(reference) / "r2splat" / "cuda" / "include"
    if not src.is_dir():
        raise FileNotFoundError(f"reference sources not found under {src}")
    sources = sorted(glob.glob(str(src / "*.cpp")) + glob.glob(str(src / "*.cu")))
    build_dir = OUT / "build"
    build_dir.mkdir(parents=True, exist_ok=True)
    if jobs:
        os.environ["MAX_JOBS"] = str(jobs)
    from torch.utils.cpp_extension import load

    load(
        name=MODULE,
        sources=sources,
        extra_include_paths=[str(inc)],
        extra_cflags=["-O3", "-std=c++17"],
        extra_cuda_cflags=[
            "-O3", "--use_fast_math", "-std=c++17", "--expt-relaxed-constexpr",
            "-gencode", "arch=compute_100a,code=sm_100a",
        ],
        build_directory=str(build_dir),
        verbose=verbose,
        is_python_module=False,
    )
    produced = sorted(build_dir.glob(MODULE + "*.so"))
    if not produced:
        raise RuntimeError("reference build produced no shared object")
    target = OUT / produced[0].name
    shutil.copy2(produced[0], target)
    stage_package(reference)
    return target


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--reference", default=None, help=f"reference checkout (default: ${REFERENCE_ENV})")
    parser.add_argument("--jobs", type=int, default=None)
    parser.add_argument("--package-only", action="store_true", help="only stage the Python package")
    args = parser.parse_args(argv)
    root = reference_root(args.reference)
    if root is None:
        parser.error(f"give --reference or set {REFERENCE_ENV}")
    if args.package_only:
        print(stage_package(root))
        return 0
    print(build(root, args.jobs))
    return 0


if __name__ == "__main__":
    sys.exit(main())
