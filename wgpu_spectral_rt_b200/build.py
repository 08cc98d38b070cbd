"""Build script for the native library libsrt_b200.so (sm_100a).

Compiles every CUDA source with nvcc for sm_100a (`-gencode
arch=compute_100a,code=sm_100a -lineinfo`), the host C++ sources with g++,
and links them into wgpu_spectral_rt_b200/libsrt_b200.so.  Objects go to
wgpu_spectral_rt_b200/_build/.  Rebuilds only what changed (by mtime,
headers included).  Then builds the headless driver
wgpu_spectral_rt_b200/srt_render (driver/srt_render.cpp), a C++ caller of
the C ABI linked against the library.

Usage:  python -m wgpu_spectral_rt_b200.build [-v] [--force]
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
BUILD = PKG / "_build"
INCLUDE = PKG.parent / "include"
LIB = PKG / "libsrt_b200.so"
DRIVER_SRC = PKG / "driver" / "srt_render.cpp"
DRIVER = PKG / "srt_render"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                     "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
# Per-file extra flags.  The shading kernels round every multiply and add
# separately (no FMA contraction), as the WGSL reference and the CPU oracle
# do; the traversal keeps contraction for its slab tests.
FILE_FLAGS = {"render_kernels.cu": ["-fmad=false"], "trace_kernels.cu": ["-fmad=true"], "present.cu": ["-fmad=false"]}
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-Wno-unused-parameter",
             f"-I{INCLUDE}", f"-I{CSRC}", "-I/usr/local/cuda/include"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    # the system g++ (an exported CXX may point at a toolchain without the runtime libs)
    return shutil.which("g++") or "g++"


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, out: Path | None = None, build_dir: Path | None = None,
          defines: list[str] | None = None) -> Path:
    """Compiles what changed and links the library.  `out`, `build_dir` and
    `defines` (-D macros for every CUDA file) produce a variant build beside
    the default one (used to compare kernel configurations)."""
    lib = Path(out) if out else LIB
    bdir = Path(build_dir) if build_dir else BUILD
    dflags = [f"-D{d}" for d in (defines or [])]
    bdir.mkdir(parents=True, exist_ok=True)
    deps = _headers()
    jobs = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = bdir / (src.stem + ".o")
        if force or _stale(obj, src, deps):
            jobs.append([_nvcc(), *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), *dflags, "-c", str(src), "-o", str(obj)])
    for src in sorted(CSRC.glob("*.cpp")):
        obj = bdir / (src.stem + ".o")
        if force or _stale(obj, src, deps):
            jobs.append([_cxx(), *CXX_FLAGS, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        p = subprocess.run(cmd, capture_output=True, text=True)
        if p.returncode != 0:
            raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{p.stdout}\n{p.stderr}")
        if verbose and (p.stdout or p.stderr):
            print(p.stdout + p.stderr, flush=True)

    with cf.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    objs = sorted(bdir.glob("*.o"))
    if jobs or force or not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        tmp = lib.with_suffix(".so.tmp")
        run([_nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"])
        os.replace(tmp, lib)
    if out is None:
        # the headless driver: a native caller of the C ABI, beside the library
        src = DRIVER_SRC
        if force or not DRIVER.exists() or any(x.stat().st_mtime > DRIVER.stat().st_mtime
                                              for x in (src, lib, INCLUDE / "srt.h")):
            tmp = DRIVER.with_suffix(".tmp")
            run([_cxx(), "-O2", "-std=c++17", "-Wall", "-Wextra", f"-I{INCLUDE}", str(src), f"-L{PKG}",
                 "-lsrt_b200", "-Wl,-rpath,$ORIGIN", "-o", str(tmp)])
            os.replace(tmp, DRIVER)
    return lib


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--out", type=Path, default=None, help="library path (default: the package's libsrt_b200.so)")
    ap.add_argument("--build-dir", type=Path, default=None)
    ap.add_argument("-D", dest="defines", action="append", default=[], help="macro for every CUDA source")
    a = ap.parse_args(argv)
    print(build(a.verbose, a.force, a.out, a.build_dir, a.defines))
    return 0


if __name__ == "__main__":
    sys.exit(main())
