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
    block, [&]() { kernel<T>(args); }); host_launch_threaded for the kernels
    named in `threaded`."""
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
        launcher = "host_launch_threaded" if name in threaded else "host_launch"
        out.append(src[pos:j])
        out.append(f"{launcher}({cfg[0]}, {cfg[1]}, [&]() {{ {kernel}({src[e + 4:m]}); }})")
        pos = m + 1
    out.append(src[pos:])
    return "".join(out)


SANITIZE = ["-fsanitize=address,undefined", "-fno-omit-frame-pointer", "-fno-sanitize-recover=all"]


def compile_unit(d: Path, name: str, flags: list[str], threaded: tuple[str, ...] = ()) -> str:
    """Rewrites csrc/<name> into d and compiles it to an object; returns its path."""
    text = rewrite_launches((CSRC / name).read_text(), threaded)
    assert "<<<" not in text
    src = d / (name + ".cpp")
    src.write_text(f"#line 1 \"{CSRC / name}\"\n" + text)
    obj = d / (name + ".o")
    subprocess.run(["g++", "-std=c++17", "-O2", *flags, "-Wno-unknown-pragmas", "-fPIC", "-c", "-I", str(d),
                    "-I", str(CSRC), "-I", str(ORACLE), str(src), "-o", str(obj)], check=True, capture_output=True)
    return str(obj)


def shim_dir(d: Path) -> Path:
    """A directory whose cuda_runtime.h is the host shim."""
    (d / "cuda_runtime.h").write_text(f'#include "{HERE / "cuda_host_shim.h"}"\n')
    return d


def link(d: Path, objs: list[str], sources: list[Path], name: str, flags: tuple[str, ...] = ()) -> ctypes.CDLL:
    so = d / name
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", *flags, "-shared", "-fPIC", "-I", str(d),
                    "-I", str(CSRC), "-I", str(ORACLE), *objs, *[str(s) for s in sources], "-o", str(so), "-lpthread"],
                   check=True, capture_output=True)
    return ctypes.CDLL(str(so))
