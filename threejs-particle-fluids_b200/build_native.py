"""Build libpfsim.so (the CUDA solver for sm_100a) in-tree.

Compiles every csrc/*.cu with nvcc for ``sm_100a`` into ``_build/`` and links
``pfsim/libpfsim.so`` against the static CUDA runtime. Objects are rebuilt only
when a source or header is newer than the object. Run as a script or call
``build()``.
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
OUT = HERE / "pfsim" / "libpfsim.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-Xptxas",
    "-warn-spills",
    f"-I{ROOT / 'include'}",
    f"-I{CSRC}",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("pfsim: nvcc not found; the CUDA extension cannot be built")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "pfsim.h"]


# Per-file flags: the mesh setup kernels keep every double multiply and add
# separately rounded, as the reference's JavaScript arithmetic is.
EXTRA_FLAGS = {"mesh_setup.cu": ["-fmad=false"]}


def _compile(src: Path, newest_header: float, verbose: bool) -> Path:
    obj = BUILD / (src.stem + ".o")
    if obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, newest_header):
        return obj
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *EXTRA_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    if res.stderr.strip() and verbose:
        print(res.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile and link libpfsim.so; returns its path."""
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    newest_header = max(p.stat().st_mtime for p in _headers())
    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, newest_header, verbose), sources))
    newest_obj = max(o.stat().st_mtime for o in objs)
    if not OUT.exists() or OUT.stat().st_mtime < newest_obj:
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(OUT), *map(str, objs)]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link of libpfsim.so failed:\n{res.stdout}\n{res.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
