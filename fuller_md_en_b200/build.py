"""Build recipe for the B200 library and the drop-in drivers.

Compiles every CUDA source for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``) with nvcc, links ``libfullermd_cuda.so``
in-tree (``fuller_md_en_b200/_lib/``), then builds the C++ drivers
``fuller_*_gpu`` against it (``fuller_md_en_b200/_bin/``).  Run as
``python -m fuller_md_en_b200.build`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
OBJ = PKG / "_obj"
LIB_DIR = PKG / "_lib"
BIN_DIR = PKG / "_bin"
LIB = LIB_DIR / "libfullermd_cuda.so"
HOST_LIB = LIB_DIR / "libfullermd_host.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", str(ROOT / "include")]
# Per-file extra flags: the integrator's scalar arithmetic rounds like the
# reference's host code (no FMA contraction).
EXTRA = {"step.cu": ["-fmad=false"]}
CUDA_SOURCES = ["nlist.cu", "airebo.cu", "rigid.cu", "mm.cu", "step.cu", "system.cu", "abi.cu", "noalloc.cu", "surrogate.cu",
                "sg_train.cu", "sg_abi.cu", "sg_step.cu", "batch.cu", "molnlist.cu", "ljprune.cu", "rebo2.cu"]

DRIVERS = ["fuller_LJ_core_gpu", "fuller_LJ_npt_md_gpu", "fuller_LJ_npt_mmmd_gpu", "fuller_airebo_npt_md_gpu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build_cuda(verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    LIB_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "fullermd.h"]
    nv = nvcc()
    jobs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        if _stale(o, [s] + headers):
            jobs.append([nv, *ARCH, *NVCC_FLAGS, *EXTRA.get(src, []), "-c", str(s), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for fut in [ex.submit(_run, j) for j in jobs]:
            fut.result()
    objs = [OBJ / (s + ".o") for s in CUDA_SOURCES]
    if _stale(LIB, objs):
        # Static runtime: the library does not depend on whichever
        # libcudart a host process (e.g. PyTorch) happens to load.
        _run([nv, *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)])
    if verbose:
        print(f"built {LIB}")
    return LIB


def build_host(verbose: bool = False) -> None:
    """Host boundary library (CLI, files, crystal set-up) and the drivers."""
    if not HOST.exists():
        return
    BIN_DIR.mkdir(exist_ok=True)
    cxx = os.environ.get("FMD_CXX", "/usr/bin/g++")
    common = sorted(HOST.glob("fmd_host*.cpp"))
    hdrs = list(HOST.glob("*.hpp")) + [ROOT / "include" / "fullermd.h"]
    flags = ["-std=c++17", "-O2", "-Wall", "-fPIC", "-pthread", "-I", str(ROOT / "include"), "-I", str(HOST)]
    if common and _stale(HOST_LIB, common + hdrs):
        _run([cxx, *flags, "-shared", "-o", str(HOST_LIB), *map(str, common)])
    for d in DRIVERS:
        src = HOST / f"{d}.cpp"
        if not src.exists():
            continue
        out = BIN_DIR / d
        if _stale(out, [src, LIB, HOST_LIB] + hdrs):
            _run([cxx, *flags, "-o", str(out), str(src), f"-L{LIB_DIR}", "-lfullermd_host", "-lfullermd_cuda",
                  f"-Wl,-rpath,{LIB_DIR}", "-Wl,-rpath,$ORIGIN/../_lib"])
    if verbose:
        print(f"built drivers in {BIN_DIR}")


def build_oracle(verbose: bool = False) -> None:
    """Test-only checkers under oracle/ (the CPU restatement, and the
    reference shims when the reference sources are present)."""
    r = subprocess.run(["make", "-C", str(ROOT / "oracle"), "-j8", "all"], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print("built oracle")


def build_tests(verbose: bool = False) -> None:
    """Test-only CUDA code (tests/cuda/), into tests/_build/: the tensor-core
    operand self test, which is not part of the product library."""
    src = ROOT / "tests" / "cuda" / "umma_selftest.cu"
    if not src.exists():
        return
    out_dir = ROOT / "tests" / "_build"
    out_dir.mkdir(exist_ok=True)
    out = out_dir / "libfmd_umma_selftest.so"
    if _stale(out, [src, CSRC / "umma.cuh"]):
        _run([nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(CSRC), "-shared", "-cudart", "static", "-o", str(out), str(src)])
    if verbose:
        print(f"built {out}")


def build_all(verbose: bool = False) -> None:
    build_cuda(verbose)
    build_host(verbose)
    build_tests(verbose)
    build_oracle(verbose)


if __name__ == "__main__":
    build_all(verbose=True)
    sys.exit(0)
