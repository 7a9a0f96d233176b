"""Build libqmbed_b200.so in place for sm_100a with nvcc.

Each CUDA translation unit under ``csrc/`` is compiled to an object in
``_build/`` (parallel nvcc processes, skipped when up to date) and linked
into ``qmbed_b200/libqmbed_b200.so`` next to this file, so the library
travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
BUILD = ROOT / "_build"
LIBRARY = PACKAGE / "libqmbed_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC,-fvisibility=hidden",
    "-Xptxas",
    "-O3",
]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list((ROOT / "include").glob("*.h")))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(dep.stat().st_mtime > mtime for dep in deps)


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    BUILD.mkdir(exist_ok=True)
    compiler = nvcc()
    hdrs = headers()
    flags = FLAGS + list(extra_flags or [])

    def compile_one(src: Path) -> Path:
        obj = BUILD / (src.stem + ".o")
        if _stale(obj, [src, *hdrs, Path(__file__)]):
            cmd = [compiler, *ARCH, *flags, "-I", str(ROOT / "include"), "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            result = subprocess.run(cmd, capture_output=True, text=True)
            if result.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src.name}:\n{result.stdout}\n{result.stderr}")
            if verbose and result.stderr:
                print(result.stderr, flush=True)
        return obj

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objects = list(pool.map(compile_one, sources()))
    if _stale(LIBRARY, objects):
        cmd = [compiler, *ARCH, "-shared", "-cudart", "static", "-o", str(LIBRARY), *map(str, objects), "-lcusolver"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIBRARY


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIBRARY)
