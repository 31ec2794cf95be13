"""The shared-reciprocal division of the exact arithmetic (physics.cuh:
MdDiv, Markstein's correction on a reciprocal refined from the hardware
seed) against IEEE division: wherever its guard holds, the quotient's bits
equal a / b's.  The exact stage kernels divide through it and fall back to
IEEE division where the guard fails, so their results stay the reference's
bit for bit.  tests/division_check.cu draws random operands over a wider
range than the guard accepts, plus all-ones and power-of-two significands,
signed zeros and dividends next to the divisor."""
import os
import re
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = ROOT / "resistivemhd_gpu_b200" / "csrc"


def _parse(out: str):
    m = re.search(r"checked (\d+) accepted (\d+) mismatches (\d+)", out)
    assert m, out
    return tuple(int(v) for v in m.groups())


def test_division_host_emulated_seed(tmp_path):
    from host_build import shim_dir

    shim_dir(tmp_path)
    exe = tmp_path / "division_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-DRMHD_HOST_EMULATION", "-x", "c++",
                    "-I", str(tmp_path), "-I", str(CSRC), str(HERE / "division_check.cu"), "-o", str(exe)],
                   check=True, capture_output=True)
    for seed in (1, 2):
        n, ok, bad = _parse(subprocess.run([str(exe), "3000000", str(seed)], check=True, capture_output=True,
                                           text=True).stdout)
        assert bad == 0
        assert ok > n // 3     # the guard accepts the bulk of the operands


@pytest.mark.gpu
def test_division_hardware_seed(gpu, tmp_path):
    """Built with nvcc for sm_100a without contraction, as the exact stage
    unit is, and run over 2^28 operand pairs per seed on the GPU."""
    exe = tmp_path / "division_check"
    nvcc = os.environ.get("NVCC", "nvcc")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-fmad=false",
                    "-I", str(CSRC), str(HERE / "division_check.cu"), "-o", str(exe)], check=True,
                   capture_output=True)
    for seed in (11, 12):
        n, ok, bad = _parse(subprocess.run([str(exe), str(1 << 28), str(seed)], check=True, capture_output=True,
                                           text=True, timeout=600).stdout)
        assert n == 1 << 28
        assert bad == 0
        assert ok > n // 3
