"""Build librmhd2d.so (the CUDA path and its C ABI) in-tree for sm_100a.

    python -m resistivemhd_gpu_b200.build        # or resistivemhd_gpu_b200.build.build()

Each translation unit is compiled by nvcc with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3``; the exact stage
kernel, the boundary/CFL kernels and the host API are compiled with
``-fmad=false`` (no fused multiply-add, so they round as the reference's
IEEE binary64 host build does), the fast stage kernel with FMA contraction,
the FP32-bulk stage kernel with --use_fast_math (single-precision operations
only; its FP64 parts round as in the fast kernel).
The CUDA runtime is linked statically and the driver API is reached through
cudaGetDriverEntryPoint, so the library loads on machines without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
OBJ = PKG / "_build"
LIB = PKG / "librmhd2d.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I", str(CSRC), "-I", str(ROOT / "include")]
UNITS = {
    "stage_exact.cu": ["-fmad=false"],
    "stage_fast.cu": ["-fmad=true"],
    "stage_bulk32.cu": ["-fmad=true", "--use_fast_math"],
    "aux_kernels.cu": ["-fmad=false"],
    "noalloc_dt.cu": ["-fmad=false"],
    "adjoint_prep.cu": ["-fmad=false"],
    "contact.cu": ["-fmad=false"],
    "adjoint.cu": ["-fmad=true"],
    "api.cu": ["-fmad=false"],
}


# A test build of the library (tests/test_gpu_wait_expiry.py): the stage
# units compiled with RMHD_TEST_WAIT_EXPIRY issue no tile load, so every
# CTA's bounded wait for its tile expires; the other units are the product's.
WAIT_TEST_DIR = ROOT / "tests" / "_build"
WAIT_TEST_LIB = WAIT_TEST_DIR / "librmhd2d_waittest.so"
STAGE_UNITS = ("stage_exact.cu", "stage_fast.cu", "stage_bulk32.cu")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*")) + [ROOT / "include" / "rmhd2d.h", Path(__file__)]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    deps = _deps()
    if not _stale(LIB, deps) and not ptxas_info:
        return LIB
    OBJ.mkdir(exist_ok=True)
    cmds = []
    for unit, extra in UNITS.items():
        obj = OBJ / (Path(unit).stem + ".o")
        cmd = ["nvcc", *ARCH, *COMMON, *extra, "-c", str(CSRC / unit), "-o", str(obj)]
        if ptxas_info:
            cmd[1:1] = ["-Xptxas", "-v"]
        cmds.append((obj, cmd))

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 4)) as pool:
        outs = list(pool.map(run, [c for _, c in cmds]))
    if verbose or ptxas_info:
        for o in outs:
            if o.strip():
                print(o, file=sys.stderr)
    link = ["nvcc", *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *[str(o) for o, _ in cmds]]
    run(link)
    return LIB


def build_wait_test(verbose: bool = False) -> Path:
    """tests/_build/librmhd2d_waittest.so (after build())."""
    deps = _deps() + [LIB]
    if not _stale(WAIT_TEST_LIB, deps):
        return WAIT_TEST_LIB
    WAIT_TEST_DIR.mkdir(parents=True, exist_ok=True)
    objs = []
    cmds = []
    for unit, extra in UNITS.items():
        if unit in STAGE_UNITS:
            obj = WAIT_TEST_DIR / (Path(unit).stem + "_waittest.o")
            cmds.append(["nvcc", *ARCH, *COMMON, *extra, "-DRMHD_TEST_WAIT_EXPIRY", "-c", str(CSRC / unit), "-o",
                         str(obj)])
        else:
            obj = OBJ / (Path(unit).stem + ".o")
        objs.append(str(obj))

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")

    with cf.ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        list(pool.map(run, cmds))
    run(["nvcc", *ARCH, "-shared", "-cudart", "static", "-o", str(WAIT_TEST_LIB), *objs])
    for o in objs:
        if o.endswith("_waittest.o"):
            Path(o).unlink()
    return WAIT_TEST_LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
    build_wait_test()
    print(LIB)
