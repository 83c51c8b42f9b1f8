"""Build the native parts in-tree.

  * detray_b200/_lib/libdetray_b200.so  - the sm_100a propagation library
                                           (nvcc, -gencode arch=compute_100a,
                                           code=sm_100a)
  * tests/native/libcore_host.so         - test-only host build of the core
  * oracle/_ref/libdetray_ref_{f64,f32}.so - the reference oracle, only when a
                                           reference checkout is present

Run: python -m detray_b200.build [--no-oracle]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "_lib" / "libdetray_b200.so"
CORE_HOST = REPO / "tests" / "native" / "libcore_host.so"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "--expt-relaxed-constexpr"]


def _newer(target: Path, sources) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(Path(s).stat().st_mtime <= t for s in sources)


def _sources():
    return ([CSRC / "dprop_api.cu"] + sorted((CSRC / "core").glob("*"))
            + [REPO / "include" / "detray_b200" / "dprop.h"])


def nvcc() -> str:
    for cand in [shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]:
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and _newer(LIB, _sources()):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc(), *NVCC_FLAGS, f"-I{REPO / 'include'}", f"-I{CSRC}",
           str(CSRC / "dprop_api.cu"), "-o", str(LIB)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


def build_core_host(force: bool = False) -> Path:
    src = REPO / "tests" / "native" / "core_host.cpp"
    if not force and _newer(CORE_HOST, [src] + _sources()):
        return CORE_HOST
    cuda_inc = Path(nvcc()).resolve().parent.parent / "include"
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared",
           f"-I{REPO / 'include'}", f"-I{CSRC}", f"-I{cuda_inc}", str(src),
           "-o", str(CORE_HOST)]
    subprocess.run(cmd, check=True)
    return CORE_HOST


def build_oracle(ref: Path | None = None) -> bool:
    """Compile the reference oracle if the reference checkout exists."""
    ref = ref or Path(os.environ.get("DETRAY_REF", "/root/reference"))
    if not (ref / "core" / "include" / "detray").exists():
        return False
    subprocess.run(["make", "-C", str(REPO / "oracle" / "ref"), f"REF={ref}"],
                   check=True)
    return True


def main(argv=None) -> None:
    argv = sys.argv[1:] if argv is None else argv
    build_library(force="--force" in argv, verbose="-v" in argv)
    build_core_host(force="--force" in argv)
    if "--no-oracle" not in argv:
        build_oracle()


if __name__ == "__main__":
    main()
