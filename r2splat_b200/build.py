"""Builds the sm_100a CUDA library ``_lib/libr2splat_b200.so`` in-tree.

Each ``csrc/*.cu`` translation unit is compiled by nvcc in parallel, then linked
into one shared object with the CUDA runtime linked statically, so the library
only needs the NVIDIA driver at run time. The flags match the numerics the
operators are specified against: ``--use_fast_math`` (the reference build's
flag, which fixes the rounding of the projection and of the contribution
thresholds), ``-O3``, and an explicit ``-gencode arch=compute_100a,code=sm_100a``.

Usage: ``python -m r2splat_b200.build [--force] [--jobs N]``.
"""

from __future__ import annotations

import argparse
import concurrent.futures
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
INCLUDE = ROOT / "include"
LIB_DIR = HERE / "_lib"
OBJ_DIR = LIB_DIR / "obj"
LIB_NAME = "libr2splat_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "--use_fast_math", "-std=c++17", "-lineinfo",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    candidate = Path(cuda_home) / "bin" / "nvcc"
    return str(candidate) if candidate.exists() else (shutil.which("nvcc") or "nvcc")


def library_path() -> Path:
    return LIB_DIR / LIB_NAME


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _fingerprint() -> str:
    digest = hashlib.sha256()
    digest.update(" ".join(NVCC_FLAGS).encode())
    for path in sorted(list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))):
        digest.update(path.name.encode())
        digest.update(path.read_bytes())
    return digest.hexdigest()


def _object_fingerprint(source: Path, extra: list[str]) -> str:
    """Flags, the translation unit and every header it may include (all of csrc/*.cuh and include/*.h)."""
    digest = hashlib.sha256()
    digest.update(" ".join(NVCC_FLAGS + extra).encode())
    digest.update(source.read_bytes())
    for path in sorted(list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))):
        digest.update(path.name.encode())
        digest.update(path.read_bytes())
    return digest.hexdigest()


def _compile(source: Path, extra: list[str]) -> Path:
    """Compiles one translation unit unless its object is up to date with its fingerprint."""
    obj = OBJ_DIR / (source.stem + ".o")
    stamp = OBJ_DIR / (source.stem + ".o.stamp")
    fingerprint = _object_fingerprint(source, extra)
    if obj.exists() and stamp.exists() and stamp.read_text() == fingerprint:
        return obj
    cmd = [nvcc(), *NVCC_FLAGS, *extra, f"-I{INCLUDE}", "-c", str(source), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{proc.stdout}\n{proc.stderr}")
    if proc.stderr.strip():
        sys.stderr.write(proc.stderr)
    stamp.write_text(fingerprint)
    return obj


def build(force: bool = False, jobs: int | None = None, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compiles and links the library unless an up-to-date build exists."""
    extra = list(extra or [])
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    stamp = LIB_DIR / "build.stamp"
    fingerprint = _fingerprint() + " ".join(extra)
    lib = library_path()
    if not force and lib.exists() and stamp.exists() and stamp.read_text() == fingerprint:
        return lib
    sources = _sources()
    workers = jobs or min(len(sources), os.cpu_count() or 4)
    if force:
        for source in sources:
            (OBJ_DIR / (source.stem + ".o.stamp")).unlink(missing_ok=True)
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as pool:
        objects = list(pool.map(lambda s: _compile(s, extra), sources))
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-cudart", "static", *[str(o) for o in objects], "-o", str(tmp)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{proc.stdout}\n{proc.stderr}")
    os.replace(tmp, lib)
    stamp.write_text(fingerprint)
    if verbose:
        print(f"built {lib}")
    return lib


def main(argv=None) -> int:
    parser = argparse.ArgumentParser(description="Build the r2splat_b200 CUDA library")
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--jobs", type=int, default=None)
    args = parser.parse_args(argv)
    print(build(force=args.force, jobs=args.jobs, verbose=True))
    return 0


if __name__ == "__main__":
    sys.exit(main())
