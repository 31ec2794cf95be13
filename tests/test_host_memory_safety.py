"""Memory safety on the CPU: the host build of the whole C ABI, every
kernel and api.cu included, runs under the address and undefined-behaviour
sanitizers (tests/host_sanitized_run.py) in a child process that preloads
the sanitizer runtime."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


def _asan_runtime() -> str | None:
    r = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True, text=True)
    path = r.stdout.strip()
    return path if r.returncode == 0 and os.path.isabs(path) and os.path.exists(path) else None


def test_host_built_kernels_stay_in_bounds():
    rt = _asan_runtime()
    if rt is None:
        pytest.skip("no address-sanitizer runtime on this host")
    env = dict(os.environ, LD_PRELOAD=rt, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1",
               UBSAN_OPTIONS="halt_on_error=1:print_stacktrace=1")
    r = subprocess.run([sys.executable, str(HERE / "host_sanitized_run.py")], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), (r.stdout[-2000:], r.stderr[-4000:])
