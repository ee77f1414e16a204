"""Build libhase_b200.so in-tree with nvcc for sm_100a."""

from __future__ import annotations

import os
import subprocess
from pathlib import Path

PACKAGE_DIR = Path(__file__).resolve().parent
REPO_ROOT = PACKAGE_DIR.parent
SOURCES = [PACKAGE_DIR / "csrc" / "hase_b200.cu", PACKAGE_DIR / "csrc" / "hase_forward.cu",
           PACKAGE_DIR / "csrc" / "hase_proposal.cu"]
HEADERS = [PACKAGE_DIR / "csrc" / "hase_device.cuh", PACKAGE_DIR / "csrc" / "hase_host.cuh",
           REPO_ROOT / "include" / "hase_b200.h", REPO_ROOT / "include" / "hase_b200_forward.h",
           REPO_ROOT / "include" / "hase_b200_proposal.h", REPO_ROOT / "include" / "hase_b200_batch.h",
           PACKAGE_DIR / "csrc" / "hase_mlp.cuh"]
LIB_PATH = PACKAGE_DIR / "libhase_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(home) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def needs_build() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB_PATH
    cmd = [nvcc(), *NVCC_FLAGS, f"-I{REPO_ROOT / 'include'}", "-o", str(LIB_PATH), *map(str, SOURCES)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB_PATH


if __name__ == "__main__":
    build_library(force=True, verbose=True)
