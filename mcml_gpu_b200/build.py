"""Build recipe for the mcml_b200 library (sm_100a) and its MCML_GPU CLI.

Compiles every source under ``csrc/`` with nvcc for ``sm_100a`` into
``lib/libmcml_b200.so`` (the C ABI of ``include/mcml_b200.h``) and links the
command-line driver ``bin/MCML_GPU`` against it.  Objects go to ``_build/``.
Rebuilds only what changed.  Usable as ``python -m mcml_gpu_b200.build``.
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
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libmcml_b200.so"
CLI = PKG / "bin" / "MCML_GPU"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Device code keeps nvcc's defaults (-fmad=true, IEEE division and sqrt):
# the walk must round exactly like the reference compiled by the same nvcc.
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-I", str(ROOT / "include"),
]

LIB_SOURCES = ["kernels.cu", "capi.cu", "config.cpp", "writers.cpp", "noalloc.cu", "batch.cu",
               "wmc.cu", "mlp.cu", "checkpoint.cpp", "order.cu", "probes.cu"]
HEADERS = ["photon.cuh", "kernels.h", "internal.h", "json_min.h", "params.h"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed ({res.returncode}): {' '.join(cmd)}\n"
                           f"{res.stdout}\n{res.stderr}")


def build(verbose: bool = False) -> Path:
    """Compile the library and CLI; returns the path of the shared library."""
    nvcc = _nvcc()
    BUILD.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    CLI.parent.mkdir(parents=True, exist_ok=True)
    common = [CSRC / h for h in HEADERS] + [ROOT / "include" / "mcml_b200.h",
                                            Path(__file__)]
    sources = [s for s in LIB_SOURCES if (CSRC / s).exists()]
    jobs = []
    objs = []
    for src in sources:
        obj = BUILD / (src.replace(".", "_") + ".o")
        objs.append(obj)
        if _stale(obj, [CSRC / src] + common):
            jobs.append([nvcc, *NVCC_FLAGS, "-c", str(CSRC / src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        for fut in [ex.submit(_run, j) for j in jobs]:
            fut.result()
    if jobs or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs)])
    cli_obj = BUILD / "cli_cpp.o"
    if _stale(cli_obj, [CSRC / "cli.cpp", ROOT / "include" / "mcml_b200.h"]):
        _run([nvcc, *NVCC_FLAGS, "-c", str(CSRC / "cli.cpp"), "-o", str(cli_obj)])
    if _stale(CLI, [cli_obj, LIB]):
        _run([nvcc, *ARCH, "-o", str(CLI), str(cli_obj), "-L", str(LIB.parent),
              "-lmcml_b200", "-Xlinker", "-rpath,$ORIGIN/../lib"])
    if verbose:
        print(f"built {LIB}\nbuilt {CLI}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
