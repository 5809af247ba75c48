"""In-tree build of ``jaccpot_b200/_lib/libjaccpot_b200.so`` for sm_100a.

One shared library holds the C ABI of include/jaccpot_b200.h: the CUDA pass
kernels (one translation unit per expansion order, compiled in parallel) and
the host-side tree/list builder.  The CUDA runtime is linked statically so the
library only needs the driver at run time.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

from . import _tables

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
OUT_DIR = HERE / "_lib"
OBJ_DIR = HERE / "_lib" / "obj"
LIB = OUT_DIR / "libjaccpot_b200.so"
ORDERS = tuple(range(1, 11))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-I", str(INCLUDE),
]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _cxx() -> str:
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("no g++ found")


def _deps(src: Path) -> list[Path]:
    return [src, *sorted(CSRC.glob("*.cuh")), *sorted((CSRC / "generated").glob("*.h")),
            INCLUDE / "jaccpot_b200.h", CSRC / "tree_build.h"]


def _stale(obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    _tables.generate(CSRC / "generated" / "bu_tables.h")
    _tables.generate_kfold(CSRC / "generated" / "kfold_tables.h")
    _tables.generate_tc(CSRC / "generated" / "tc_plans.h")
    _tables.generate_bu_code(CSRC / "generated" / "bu_code.h")
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    jobs_todo = []
    for p in ORDERS:
        obj = OBJ_DIR / f"fmm_order_p{p}.o"
        src = CSRC / "fmm_order.cu"
        if _stale(obj, _deps(src)):
            jobs_todo.append([nvcc, *NVCC_FLAGS, f"-DJB_ORDER={p}", "-c", str(src), "-o", str(obj)])
    for name in ("fmm_capi", "fmm_noalloc", "fmm_gears", "m2l_tc"):
        src = CSRC / f"{name}.cu"
        if not src.exists():
            continue
        obj = OBJ_DIR / f"{name}.o"
        if _stale(obj, _deps(src)):
            jobs_todo.append([nvcc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    # The device tree build reproduces the host builder's FP64 arithmetic
    # operation for operation, so nothing in it may be contracted into an FMA.
    tg_src, tg_obj = CSRC / "tree_gpu.cu", OBJ_DIR / "tree_gpu.o"
    if _stale(tg_obj, [tg_src, CSRC / "dev_prims.cuh", INCLUDE / "jaccpot_b200.h"]):
        jobs_todo.append([nvcc, *NVCC_FLAGS, "-fmad=false", "-c", str(tg_src), "-o", str(tg_obj)])
    sg_src, sg_obj = CSRC / "schedule_gpu.cu", OBJ_DIR / "schedule_gpu.o"
    if _stale(sg_obj, [sg_src, CSRC / "dev_prims.cuh", INCLUDE / "jaccpot_b200.h"]):
        jobs_todo.append([nvcc, *NVCC_FLAGS, "-c", str(sg_src), "-o", str(sg_obj)])
    tb_obj = OBJ_DIR / "tree_build.o"
    if _stale(tb_obj, _deps(CSRC / "tree_build.cpp")):
        jobs_todo.append([_cxx(), "-O3", "-fopenmp", "-fPIC", "-std=c++17", "-I", str(INCLUDE),
                          "-c", str(CSRC / "tree_build.cpp"), "-o", str(tb_obj)])
    if jobs_todo:
        n = jobs or max(1, min(len(jobs_todo), os.cpu_count() or 4))
        with cf.ThreadPoolExecutor(n) as ex:
            list(ex.map(_run, jobs_todo))
    objs = sorted(str(o) for o in OBJ_DIR.glob("*.o"))
    if not LIB.exists() or any(Path(o).stat().st_mtime > LIB.stat().st_mtime for o in objs):
        _run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(LIB), *objs,
              "-Xcompiler", "-fopenmp", "-lgomp"])
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
