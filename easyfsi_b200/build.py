"""Build recipe of the easyfsi_b200 CUDA library (sm_100a).

``python -m easyfsi_b200.build`` compiles every ``csrc/*.cu`` with nvcc into
``easyfsi_b200/libeasyfsi_b200.so`` (in-tree, so it travels with the source
tree).  The library exports the C ABI declared in ``include/easyfsi_b200.h``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_DIR = PACKAGE_DIR.parent
CSRC_DIR = PACKAGE_DIR / "csrc"
INCLUDE_DIR = REPO_DIR / "include"
LIB_PATH = PACKAGE_DIR / "libeasyfsi_b200.so"
BUILD_DIR = PACKAGE_DIR / "_build"

NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
]


# Per-source extra flags.  The node search keeps the reference's f32
# expressions unfused, so its geometry rounds as the expressions read.
EXTRA_FLAGS = {"efsi_ibsearch.cu": ["-fmad=false"]}


def _nvcc() -> str:
    candidates = [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]
    for cand in candidates:
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the easyfsi_b200 CUDA library cannot be built")


def _host_compiler() -> list[str]:
    # nvcc needs a host g++ that it supports; prefer the system one.
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return ["-ccbin", cand]
    return []


def sources() -> list[Path]:
    return sorted(CSRC_DIR.glob("*.cu"))


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    built = LIB_PATH.stat().st_mtime
    deps = sources() + sorted(CSRC_DIR.glob("*.cuh")) + sorted(INCLUDE_DIR.glob("*.h"))
    return any(dep.stat().st_mtime > built for dep in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library if a source changed (or ``force``); return its path."""
    if not force and not _stale():
        return LIB_PATH
    nvcc = _nvcc()
    BUILD_DIR.mkdir(exist_ok=True)
    objects = []
    for src in sources():
        obj = BUILD_DIR / (src.stem + ".o")
        cmd = [nvcc, *_host_compiler(), *NVCC_FLAGS, *EXTRA_FLAGS.get(src.name, []), f"-I{INCLUDE_DIR}", "-c",
               str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objects.append(str(obj))
    tmp = LIB_PATH.with_suffix(".so.tmp")
    link = [nvcc, *_host_compiler(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objects, "-o", str(tmp)]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    path = build(force="--force" in sys.argv, verbose=True)
    print(path)
