"""Build recipe for the reference's own step, used as test oracle and baseline.

TEST INFRASTRUCTURE ONLY.  Compiles the UNMODIFIED single-GPU library of
keita-akutagawa/ResistiveMHD_GPU from the sources where they lie (read-only)
together with the project-written driver ``oracle/ref_driver.cu``:

* ``oracle/_ref/ref_gpu_{periodic,symmetric}`` -- nvcc, sm_100a, the flags of
  the reference's example makefiles (``-O3 -rdc=true``) with the arch swapped
  and the MSVC-only ``-Xcompiler "/wd 4819"`` dropped
  (ResistiveMHD_singleGPU_thrust/examples2D/plasmoid/makefile:2).
* ``oracle/_ref/ref_cpu_{periodic,symmetric}`` -- g++ with OpenMP against
  Thrust's OMP backend.  Each library source is read, its kernel-launch syntax
  ``k<<<g, b>>>(args)`` is rewritten in memory to
  ``host_launch(g, b, [&]() { k(args); })`` and the text is piped to the
  compiler on stdin; nothing of the reference is written to disk.  No
  arithmetic is edited.

* ``oracle/_ref/mc_host`` -- the CT-Contact and wall parts of the multi-GPU
  library (ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU: const.cu, ct.cu,
  boundary.cu, mpi.cu, sign.cu), unmodified, with the project-written driver
  ``oracle/mc_driver.cu``, built the same way for the host on one rank: its
  ``#include <mpi.h>`` (mpi.hpp) finds the single-rank stand-in
  ``oracle/mpi_stub/mpi.h`` first on the include path.

Outputs go only to ``oracle/_ref/`` (git-ignored; it travels to the GPU box).
When the reference tree is absent (the GPU box) nothing is built.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF_ROOT = Path(os.environ.get("RMHD_REFERENCE_ROOT", "/root/reference"))
LIBS = {
    "periodic": "ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_periodicXY",
    "symmetric": "ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_symmetricXY",
}
CUDA_INC = "/usr/local/cuda/include"
GENCODE = "-gencode=arch=compute_100a,code=sm_100a"

_LAUNCH = re.compile(r"([A-Za-z_]\w*)\s*<<<(.*?)>>>\s*\(", re.S)


def rewrite_launches(src: str) -> str:
    """Rewrite every ``k<<<g, b>>>(args)`` into a host_launch call."""
    out = []
    pos = 0
    for m in _LAUNCH.finditer(src):
        if m.start() < pos:
            continue
        depth, k = 1, m.end()
        while depth:
            c = src[k]
            depth += (c == "(") - (c == ")")
            k += 1
        args = src[m.end():k - 1]
        out.append(src[pos:m.start()])
        out.append(f"host_launch({m.group(2)}, [&]() {{ {m.group(1)}({args}); }})")
        pos = k
    out.append(src[pos:])
    return "".join(out)


def _run(cmd, stdin_text=None):
    r = subprocess.run(cmd, input=stdin_text, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def _gpu_objects(name: str, libdir: Path, objdir: Path, pool) -> list:
    jobs = []
    for src in sorted(libdir.glob("*.cu")):
        obj = objdir / (src.stem + ".o")
        cmd = ["nvcc", "-O3", GENCODE, "-rdc=true", "-I", str(libdir), "-c", str(src), "-o", str(obj)]
        jobs.append((obj, pool.submit(_run, cmd)))
    obj = objdir / "ref_driver.o"
    defs = ["-DREF_SYMMETRIC"] if name == "symmetric" else []
    cmd = ["nvcc", "-O3", GENCODE, "-rdc=true", *defs, "-I", str(libdir), "-x", "cu", "-c",
           str(HERE / "ref_driver.cu"), "-o", str(obj)]
    jobs.append((obj, pool.submit(_run, cmd)))
    return jobs


def _cpu_objects(name: str, libdir: Path, objdir: Path, pool) -> list:
    common = ["g++", "-O3", "-fopenmp", "-std=c++17", "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_OMP",
              "-DREF_HOST_BUILD", "-include", str(HERE / "ref_host_shim.h"), "-I", str(libdir),
              "-I", CUDA_INC, "-w"]
    jobs = []
    for src in sorted(libdir.glob("*.cu")):
        obj = objdir / (src.stem + ".o")
        text = rewrite_launches(src.read_text())
        cmd = common + ["-x", "c++", "-c", "-", "-o", str(obj)]
        jobs.append((obj, pool.submit(_run, cmd, text)))
    obj = objdir / "ref_driver.o"
    defs = ["-DREF_SYMMETRIC"] if name == "symmetric" else []
    text = (HERE / "ref_driver.cu").read_text()
    shim_defs = ("thread_local ref_uint3 blockIdx; thread_local ref_uint3 threadIdx; "
                 "thread_local dim3 blockDim; thread_local dim3 gridDim;\n")
    cmd = common + defs + ["-x", "c++", "-c", "-", "-o", str(obj)]
    jobs.append((obj, pool.submit(_run, cmd, text + "\n" + shim_defs)))
    return jobs


MC_LIB = "ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU"
MC_SOURCES = ("const.cu", "ct.cu", "boundary.cu", "mpi.cu", "sign.cu")


def mc_binary() -> Path:
    return OUT / "mc_host"


def build_mc(verbose=True) -> bool:
    """Build oracle/_ref/mc_host; returns False when the reference is absent."""
    libdir = REF_ROOT / MC_LIB
    if not libdir.is_dir():
        return False
    OUT.mkdir(parents=True, exist_ok=True)
    target = mc_binary()
    deps = [libdir / f for f in MC_SOURCES] + list(libdir.glob("*.hpp")) + [
        HERE / f for f in ("mc_driver.cu", "ref_host_shim.h", "build_ref.py")] + [HERE / "mpi_stub" / "mpi.h"]
    if target.exists() and target.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return True
    objdir = OUT / "obj_mc"
    objdir.mkdir(parents=True, exist_ok=True)
    common = ["g++", "-O3", "-fopenmp", "-std=c++17", "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_OMP",
              "-DREF_HOST_BUILD", "-include", str(HERE / "ref_host_shim.h"), "-I", str(HERE / "mpi_stub"),
              "-I", str(libdir), "-I", CUDA_INC, "-w"]
    shim_defs = ("thread_local ref_uint3 blockIdx; thread_local ref_uint3 threadIdx; "
                 "thread_local dim3 blockDim; thread_local dim3 gridDim;\n")
    objs = []
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        jobs = []
        for name in MC_SOURCES:
            obj = objdir / (Path(name).stem + ".o")
            text = rewrite_launches((libdir / name).read_text())
            jobs.append((obj, pool.submit(_run, common + ["-x", "c++", "-c", "-", "-o", str(obj)], text)))
        obj = objdir / "mc_driver.o"
        text = rewrite_launches((HERE / "mc_driver.cu").read_text()) + "\n" + shim_defs
        jobs.append((obj, pool.submit(_run, common + ["-x", "c++", "-c", "-", "-o", str(obj)], text)))
        for obj, fut in jobs:
            fut.result()
            objs.append(str(obj))
    _run(["g++", "-O3", "-fopenmp", *objs, "-o", str(target)])
    shutil.rmtree(objdir, ignore_errors=True)
    if verbose:
        print(f"[build_ref] built {target.relative_to(HERE.parent)}", file=sys.stderr)
    return True


def build(which=("gpu", "cpu"), verbose=True) -> bool:
    """Build the reference binaries; returns False when the reference is absent."""
    if not REF_ROOT.is_dir():
        if verbose:
            print(f"[build_ref] reference tree {REF_ROOT} absent; using prebuilt oracle/_ref", file=sys.stderr)
        return False
    OUT.mkdir(parents=True, exist_ok=True)
    links = []
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        for name, rel in LIBS.items():
            libdir = REF_ROOT / rel
            for kind in which:
                target = OUT / f"ref_{kind}_{name}"
                objdir = OUT / f"obj_{kind}_{name}"
                if target.exists() and target.stat().st_mtime >= max(
                        [p.stat().st_mtime for p in libdir.glob("*")] +
                        [(HERE / f).stat().st_mtime for f in ("ref_driver.cu", "ref_host_shim.h", "build_ref.py")]):
                    continue
                objdir.mkdir(parents=True, exist_ok=True)
                jobs = (_gpu_objects if kind == "gpu" else _cpu_objects)(name, libdir, objdir, pool)
                links.append((kind, target, objdir, jobs))
        for kind, target, objdir, jobs in links:
            objs = []
            for obj, fut in jobs:
                fut.result()
                objs.append(str(obj))
            if kind == "gpu":
                cmd = ["nvcc", "-O3", GENCODE, "-rdc=true", *objs, "-o", str(target)]
            else:
                cmd = ["g++", "-O3", "-fopenmp", *objs, "-o", str(target)]
            _run(cmd)
            shutil.rmtree(objdir, ignore_errors=True)
            if verbose:
                print(f"[build_ref] built {target.relative_to(HERE.parent)}", file=sys.stderr)
    return True


if __name__ == "__main__":
    kinds = tuple(sys.argv[1:]) or ("gpu", "cpu", "mc")
    build(tuple(k for k in kinds if k != "mc"))
    if "mc" in kinds:
        build_mc()
