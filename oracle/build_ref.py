"""Build recipe for the reference CUDA extension used as a parity checker.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module.

Compiles the reference's own low-level operator sources (``r2splat/cuda/csrc``
of MedAPT-group/R2Splat, the files listed by its ``setup.py:17-22``) unmodified,
from where they lie, with the reference's nvcc flags (``setup.py:29-34``:
``-O3 --use_fast_math -std=c++17 --expt-relaxed-constexpr``) plus an explicit
``sm_100a`` target. The product is a torch extension module named
``r2splat_ref_csrc`` written to ``oracle/_ref/``; intermediate objects go to
``oracle/_ref/build/``. The module exposes the reference's 40 pybind names
(``ext.cpp:8-183``) so GPU parity tests and the reference bench arm can call the
reference kernels on the same inputs as this package.

Usage (needs the reference checkout, nvcc and ninja; no GPU):
    python oracle/build_ref.py [--reference PATH] [--jobs N]
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
MODULE = "r2splat_ref_csrc"
DEFAULT_REFERENCE = "/root/reference"


def built_module_path() -> Path | None:
    hits = sorted(OUT.glob(MODULE + "*.so"))
    return hits[0] if hits else None


def build(reference: str = DEFAULT_REFERENCE, jobs: int | None = None, verbose: bool = True) -> Path:
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
    return target


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--reference", default=DEFAULT_REFERENCE)
    parser.add_argument("--jobs", type=int, default=None)
    args = parser.parse_args(argv)
    path = build(args.reference, args.jobs)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
