"""Build the CUDA library agal_b200/libagal_b200.so in-tree for sm_100a.

Every .cu and .cpp under agal_b200/csrc is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared
library with the CUDA runtime linked statically, so the library loads on a
machine without a GPU (it only needs libcuda when a CUDA call is made).

Usage: ``python -m agal_b200.build [--force] [-j N]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libagal_b200.so"
OBJ = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def headers() -> list[Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) +
                  list((PKG.parent / "include").glob("*.h")))


def _compile(src: Path, extra: list[str]) -> Path:
    obj = OBJ / (src.name + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra, "-I", str(PKG.parent / "include"),
           "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def up_to_date() -> bool:
    if not OUT.exists():
        return False
    t = OUT.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources() + headers() + [Path(__file__)])


def _stale(src: Path, newest_header: float) -> bool:
    obj = OBJ / (src.name + ".o")
    return not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)


def build(force: bool = False, jobs: int | None = None, verbose_ptxas: bool = False) -> Path:
    if not force and up_to_date():
        return OUT
    OBJ.mkdir(exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []
    srcs = sources()
    # Objects newer than their source and every header are reused.
    newest_header = max([p.stat().st_mtime for p in headers()] + [Path(__file__).stat().st_mtime])
    todo = [s for s in srcs if force or _stale(s, newest_header)]
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        list(ex.map(lambda s: _compile(s, extra), todo))
    objs = [OBJ / (s.name + ".o") for s in srcs]
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(OUT), *map(str, objs)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/spill report")
    a = ap.parse_args(argv)
    out = build(force=a.force or a.ptxas, jobs=a.j, verbose_ptxas=a.ptxas)
    print(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
