"""TEST INFRASTRUCTURE: builds kernel sources of resistivemhd_gpu_b200/csrc
for the host, so CPU tests can run them without a GPU.

Each `kernel<<<grid, block, smem, stream>>>(args)` launch is rewritten into
a call of tests/cuda_host_shim.h: host_launch (a loop over the launch's
blocks and threads) or, for kernels that synchronise their block,
host_launch_threaded (one host thread per CUDA thread, with a block
barrier)."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE.parent / "resistivemhd_gpu_b200" / "csrc"
ORACLE = HERE.parent / "oracle"


def _split_top_level(s: str) -> list[str]:
    parts, depth, cur = [], 0, []
    for ch in s:
        if ch in "([{":
            depth += 1
        elif ch in ")]}":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    parts.append("".join(cur).strip())
    return parts


def rewrite_launches(src: str, threaded: tuple[str, ...] = ()) -> str:
    """`kernel<T><<<grid, block, smem, stream>>>(args)` -> host_launch(grid,
    block, [=]() { kernel<T>(args); }); host_launch_threaded for the kernels
    named in `threaded`.  The arguments are captured by value, as a launch
    copies them, so a recorded launch (stream capture) replays with them."""
    out, pos = [], 0
    while True:
        k = src.find("<<<", pos)
        if k < 0:
            break
        e = src.find(">>>", k)
        j, depth = k, 0                      # the kernel expression before <<<
        while j > 0:
            ch = src[j - 1]
            if ch == ">":
                depth += 1
            elif ch == "<":
                if depth == 0:
                    break
                depth -= 1
            elif depth == 0 and not (ch.isalnum() or ch in "_:"):
                break
            j -= 1
        kernel = src[j:k]
        assert src[e + 3] == "(", src[k:e + 10]
        m, d = e + 3, 0                      # the call's argument list
        while True:
            if src[m] == "(":
                d += 1
            elif src[m] == ")":
                d -= 1
                if d == 0:
                    break
            m += 1
        cfg = _split_top_level(src[k + 3:e])
        name = kernel.split("<")[0]
        out.append(src[pos:j])
        if name in threaded:
            smem = cfg[2] if len(cfg) > 2 else "0"
            out.append(f"host_launch_threaded({cfg[0]}, {cfg[1]}, [=]() {{ {kernel}({src[e + 4:m]}); }}, {smem})")
        else:
            out.append(f"host_launch({cfg[0]}, {cfg[1]}, [=]() {{ {kernel}({src[e + 4:m]}); }})")
        pos = m + 1
    out.append(src[pos:])
    return "".join(out)


SANITIZE = ["-O1", "-fsanitize=address,undefined", "-fno-omit-frame-pointer", "-fno-sanitize-recover=all"]


def _rewrite(name: str, threaded: tuple[str, ...]) -> str:
    text = rewrite_launches((CSRC / name).read_text(), threaded)
    # dynamic shared memory: the running block's buffer of the threaded launch
    text = text.replace("extern __shared__ __align__(1024) unsigned char smem_raw[];",
                        "unsigned char *smem_raw = shim_dynamic_smem();")
    assert "<<<" not in text and "extern __shared__" not in text
    return f"#line 1 \"{CSRC / name}\"\n" + text


def compile_unit(d: Path, name: str, flags: list[str], threaded: tuple[str, ...] = (),
                 headers: tuple[str, ...] = ()) -> str:
    """Rewrites csrc/<name> into d and compiles it to an object; returns its
    path.  `headers` are csrc headers holding kernels the unit includes:
    rewritten into d too, where the unit's #include finds them first."""
    for h in headers:
        (d / h).write_text(_rewrite(h, threaded))
    src = d / (name + ".cpp")
    src.write_text(_rewrite(name, threaded))
    obj = d / (name + ".o")
    subprocess.run(["g++", "-std=c++17", "-O2", *flags, "-Wno-unknown-pragmas", "-fPIC", "-c", "-I", str(d),
                    "-I", str(CSRC), "-I", str(ORACLE), str(src), "-o", str(obj)], check=True, capture_output=True)
    return str(obj)


def shim_dir(d: Path) -> Path:
    """A directory whose cuda_runtime.h and cuda.h are the host shim."""
    (d / "cuda_runtime.h").write_text(f'#include "{HERE / "cuda_host_shim.h"}"\n')
    (d / "cuda.h").write_text(f'#include "{HERE / "cuda_host_shim.h"}"\n')
    (d / "cudaTypedefs.h").write_text(f'#include "{HERE / "cuda_host_shim.h"}"\n')
    return d


def link(d: Path, objs: list[str], sources: list[Path], name: str, flags: tuple[str, ...] = ()) -> ctypes.CDLL:
    so = d / name
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", *flags, "-shared", "-fPIC", "-I", str(d),
                    "-I", str(CSRC), "-I", str(ORACLE), *objs, *[str(s) for s in sources], "-o", str(so), "-lpthread"],
                   check=True, capture_output=True)
    return ctypes.CDLL(str(so))


EMU = "-DRMHD_HOST_EMULATION"
THREADED = ("stage_kernel", "stage_batch_kernel", "kernel", "rate_kernel", "boundary_batch_kernel",
            "dt_noalloc_kernel", "contact_flux_tiled_kernel")
OFF = ["-ffp-contract=off"]
CONTRACTED = ["-ffp-contract=fast", "-mfma"]
# each unit with the contraction nvcc gives it (resistivemhd_gpu_b200/build.py)
ABI_UNITS = {"api.cu": OFF, "stage_exact.cu": OFF, "stage_fast.cu": CONTRACTED, "stage_bulk32.cu": CONTRACTED,
             "aux_kernels.cu": OFF, "noalloc_dt.cu": OFF, "adjoint_prep.cu": OFF, "contact.cu": OFF,
             "adjoint.cu": CONTRACTED + ["-DRMHD_ADJ_HOST_RN"]}


def has_fma() -> bool:
    return " fma " in open("/proc/cpuinfo").read().replace("\n", " ")


def build_host_abi(d: Path, extra: tuple[str, ...] = ()) -> ctypes.CDLL:
    """Every unit of csrc/, api.cu included, built for the host into one
    library with the C ABI's signatures set (tests/cuda_host_runtime.h
    answers api.cu's runtime calls); `extra` adds compiler flags to every
    unit."""
    from concurrent.futures import ThreadPoolExecutor

    from resistivemhd_gpu_b200 import _lib

    shim_dir(d)
    # stage_impl.cuh is rewritten into d by each stage unit: write it once first
    compile_unit(d, "stage_exact.cu", [*OFF, EMU, "-fsyntax-only"], threaded=THREADED, headers=("stage_impl.cuh",))

    def unit(item):
        u, f = item
        return compile_unit(d, u, [*f, EMU, *extra], threaded=THREADED)

    with ThreadPoolExecutor(max_workers=8) as pool:
        objs = list(pool.map(unit, ABI_UNITS.items()))
    lib = link(d, objs, [HERE / "host_tma.cpp"], "librmhd2d_host.so", (EMU, *extra))
    for name, res, args in _lib.SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
