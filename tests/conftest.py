import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and librmhd2d.so")


def load_golden(name: str):
    """Returns (setup, initial_state, final_state, dts, total_time) of a fixture."""
    from resistivemhd_gpu_b200.setups import Setup

    z = np.load(GOLDEN / f"{name}.npz")
    dx, dy, gamma, cfl, eps, eta = (float(v) for v in z["params"])
    tab = z["eta_table"]
    s = Setup(name, z["initial"].copy(), dx, dy, gamma, cfl, eps, eta,
              tab.copy() if tab.size else None, str(z["bc"]))
    return s, z["initial"], z["final"], z["dts"], float(z["total_time"])


# runs of the reference's own build (make_golden.py); other fixtures in the
# folder (e.g. plasmoid_degenerate_face.npz) carry no "params" and have their own tests
GOLDEN_CASES = sorted(p.stem for p in GOLDEN.glob("*.npz") if "params" in np.load(p).files)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import OracleLib

    return OracleLib()


@pytest.fixture(scope="session")
def tangent():
    from oracle.oracle import TangentLib

    return TangentLib()


@pytest.fixture(scope="session")
def gpu(request, tmp_path_factory):
    """Skips nothing: a GPU test run without a usable B200 is a failure.

    With RMHD_TESTS_ON_HOST_BUILD=1 the GPU tests run instead against the
    host build of the whole C ABI (tests/host_build.py: build_host_abi),
    bound to the Python mirror for the session: a check of the sources on a
    machine without a GPU, not a measurement of the CUDA library.  Tests
    that link librmhd2d.so into their own programs, or that need torch's
    device memory, still need the GPU."""
    import ctypes
    import os

    from resistivemhd_gpu_b200 import _lib

    if os.environ.get("RMHD_TESTS_ON_HOST_BUILD") == "1":
        from host_build import build_host_abi

        mp = pytest.MonkeyPatch()
        mp.setattr(_lib, "_lib", build_host_abi(tmp_path_factory.mktemp("abihost")))
        request.addfinalizer(mp.undo)
        return _lib._lib

    lib = _lib.load()
    cudart_ok = True
    try:
        import torch

        cudart_ok = torch.cuda.is_available()
    except Exception:
        pass
    assert cudart_ok, "GPU tests need a CUDA device"
    return lib
