"""Build the native libraries of asar-focus B200.

* ``asarf/libasarf.so``: the product — CUDA kernels for sm_100a + host planner + C ABI
  (include/asarf.h).  Built with nvcc, in-tree, so it travels with the source tree.
* ``build_emu(dir)``: a test-only library that runs the same kernel bodies on the CPU
  (host emulation backend).  The CPU test suite uses it to check the kernel code against
  the oracle without a GPU; nothing in the product loads it.

Usage: python asar-focus_b200/build.py [--emu DIR]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INC = ROOT / "include"
LIB = PKG / "asarf" / "libasarf.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_INC = Path(NVCC).resolve().parent.parent / "include"

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build failed: {' '.join(cmd[:3])} ...")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp")) + sorted(CSRC.glob("*.cuh")) + \
        sorted(CSRC.glob("*.h")) + [INC / "asarf.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    """Compile the product library (sm_100a)."""
    deps = _sources()
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    common = ["-std=c++17", "-O3", "-lineinfo", f"-I{INC}", f"-I{CSRC}", "-Xcompiler", "-fPIC"]
    objs = []
    for src in ("kernels.cu", "noalloc.cu", "host.cpp", "stages.cpp", "batch.cpp", "strip.cpp", "l0.cpp"):
        obj = objdir / (src + ".o")
        cmd = [NVCC, *GENCODE, *common, "-c", str(CSRC / src), "-o", str(obj)]
        if src.endswith(".cu") and verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
        if src.endswith(".cpp"):
            cmd = [NVCC, *common, "-x", "cu", *GENCODE, "-c", str(CSRC / src), "-o", str(obj)]
        _run(cmd)
        objs.append(str(obj))
    _run([NVCC, *GENCODE, "-shared", "-o", str(LIB), *objs, "-lcudart"])
    return LIB


def build_emu(out_dir: str | os.PathLike, force: bool = False) -> Path:
    """Compile the host-emulation test library into out_dir (CPU only, no CUDA device code)."""
    out = Path(out_dir) / "libasarf_emu.so"
    deps = _sources()
    if not force and not _stale(out, deps):
        return out
    out.parent.mkdir(parents=True, exist_ok=True)
    # compiled under a per-process name and renamed into place, so that test processes
    # running side by side never load a half-written library
    tmp = out.with_name(f".{out.name}.{os.getpid()}.tmp")
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-fno-strict-aliasing", "-fPIC", "-shared", "-DASARF_HOST_EMU",
           f"-I{INC}", f"-I{CSRC}", f"-I{CUDA_INC}", "-x", "c++", str(CSRC / "host.cpp"), "-x", "c++",
           str(CSRC / "stages.cpp"), "-x", "c++", str(CSRC / "batch.cpp"), "-x", "c++", str(CSRC / "strip.cpp"), "-x", "c++",
           str(CSRC / "l0.cpp"), "-x", "c++", str(CSRC / "emu.cpp"),
           "-o", str(tmp)]
    try:
        _run(cmd)
        os.replace(tmp, out)
    finally:
        if tmp.exists():
            tmp.unlink()
    return out


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--emu":
        print(build_emu(sys.argv[2], force=True))
    else:
        print(build(force=True, verbose_ptxas="-v" in sys.argv))
