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
CORE_HOST_STEPPED = REPO / "tests" / "native" / "libcore_host_stepped.so"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "--expt-relaxed-constexpr"]


def _newer(target: Path, sources) -> bool:
    if not target.exists():
        return False
    t = target.stat().st_mtime
    return all(Path(s).stat().st_mtime <= t for s in sources)


# translation units of the library, compiled in parallel
UNITS = ["dprop_api.cu", "rounds_api.cu", "adjoint_api.cu", "fp64_api.cu",
         "direct_api.cu", "scan_api.cu"]


def _headers():
    return (sorted((CSRC / "core").glob("*")) + sorted(CSRC.glob("*.cuh"))
            + [REPO / "include" / "detray_b200" / "dprop.h"])


def _sources():
    return [CSRC / u for u in UNITS] + _headers()


def nvcc() -> str:
    for cand in [shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]:
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and _newer(LIB, _sources()):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    obj_dir = LIB.parent / "obj"
    obj_dir.mkdir(exist_ok=True)
    flags = [f for f in NVCC_FLAGS if f != "-shared"]
    procs = []
    objs = []
    for unit in UNITS:
        src = CSRC / unit
        obj = obj_dir / (src.stem + ".o")
        objs.append(obj)
        if not force and _newer(obj, [src] + _headers()):
            continue
        cmd = [nvcc(), *flags, "-c", f"-I{REPO / 'include'}", f"-I{CSRC}",
               str(src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((unit, subprocess.Popen(cmd)))
    failed = [unit for unit, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    subprocess.run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a",
                    "-shared", *[str(o) for o in objs], "-o", str(LIB)],
                   check=True)
    return LIB


def build_core_host(force: bool = False, stepped: bool = False) -> Path:
    """Host build of the core for the tests.  stepped: built with
    DPROP_NO_CYCLE_SKIP, so that exact cycles are stepped out to the path
    limit as the reference does instead of being skipped."""
    src = REPO / "tests" / "native" / "core_host.cpp"
    out = CORE_HOST_STEPPED if stepped else CORE_HOST
    if not force and _newer(out, [src] + _sources()):
        return out
    cuda_inc = Path(nvcc()).resolve().parent.parent / "include"
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared",
           f"-I{REPO / 'include'}", f"-I{CSRC}", f"-I{cuda_inc}", str(src),
           "-o", str(out)]
    if stepped:
        cmd.insert(1, "-DDPROP_NO_CYCLE_SKIP")
    subprocess.run(cmd, check=True)
    return out


def build_oracle(ref: Path | str | None = None) -> bool:
    """Compile the reference oracle from the reference checkout at ``ref``
    (or $DETRAY_REF); does nothing if neither names a checkout."""
    ref = ref or os.environ.get("DETRAY_REF")
    if not ref:
        return False
    ref = Path(ref)
    if not (ref / "core" / "include" / "detray").exists():
        return False
    subprocess.run(["make", "-C", str(REPO / "oracle" / "ref"), f"REF={ref}"],
                   check=True)
    return True


def main(argv=None) -> None:
    argv = sys.argv[1:] if argv is None else argv
    build_library(force="--force" in argv, verbose="-v" in argv)
    build_core_host(force="--force" in argv)
    refs = [a.split("=", 1)[1] for a in argv if a.startswith("--ref=")]
    if "--no-oracle" not in argv:
        build_oracle(refs[0] if refs else None)


if __name__ == "__main__":
    main()
