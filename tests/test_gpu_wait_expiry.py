"""The stage kernels' bounded wait for their staged tile, made to expire
without a fault: a test build of the library (tests/_build/
librmhd2d_waittest.so, resistivemhd_gpu_b200/build.py: build_wait_test)
compiles the stage units with RMHD_TEST_WAIT_EXPIRY, so the staging thread
arms the tile's mbarrier but issues no load and every thread gives up after
a few tries.  Nothing is then in flight when a CTA returns.  The library
must report RMHD2D_ERR_KERNEL (the reference's only failure signal is the
NaN check, resistiveMHD_2D.cu:294-309; this extends it), and the process's
CUDA context must stay usable: the product library, loaded beside it, still
steps bit for bit with the oracle.  The same path runs first on the host
build of the C ABI."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from host_build import build_host_abi, has_fma

ROOT = Path(__file__).resolve().parents[1]
WAIT_TEST_LIB = ROOT / "tests" / "_build" / "librmhd2d_waittest.so"
ERR_KERNEL = 6


def _load(path):
    from resistivemhd_gpu_b200 import _lib

    lib = ctypes.CDLL(str(path))
    for name, res, args in _lib.SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


def _expire_on(lib):
    """Steps a solver of `lib` whose stage kernels never get their tile:
    returns (status of the step, status of the following query, its text)."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(40, 36, seed=9, bc="symmetric", with_table=True)
    cfg = Solver.make_config(s.nx, s.ny, s.dx, s.dy, gamma=s.gamma, cfl=s.cfl, eps=s.eps, eta=s.eta, bc=s.bc)
    h = ctypes.c_void_p()
    assert lib.rmhd2d_create(ctypes.byref(cfg), ctypes.byref(h)) == 0
    try:
        st = np.ascontiguousarray(s.state)
        D = ctypes.POINTER(ctypes.c_double)
        assert lib.rmhd2d_set_state(h, st.ctypes.data_as(D), 1) == 0
        rc_step = lib.rmhd2d_step_rk2(h)
        crashed = ctypes.c_int()
        rc_query = lib.rmhd2d_check_crashed(h, ctypes.byref(crashed))
        text = lib.rmhd2d_last_error(h).decode()
        return rc_step, rc_query, text
    finally:
        lib.rmhd2d_destroy(h)


def test_wait_expiry_on_host_build(tmp_path):
    if not has_fma():
        pytest.skip("the host has no fused multiply-add to model the device build with")
    lib = build_host_abi(tmp_path, extra=("-DRMHD_TEST_WAIT_EXPIRY",))
    rc_step, rc_query, text = _expire_on(lib)
    assert rc_step == 0                       # the step is enqueued
    assert rc_query == ERR_KERNEL, text       # the next query reports the expired wait
    assert "bounded wait" in text


@pytest.mark.gpu
def test_wait_expiry_reports_kernel_error_and_context_survives(gpu, oracle):
    assert WAIT_TEST_LIB.exists(), "build it with resistivemhd_gpu_b200.build.build_wait_test()"
    rc_step, rc_query, text = _expire_on(_load(WAIT_TEST_LIB))
    assert rc_step == 0
    assert rc_query == ERR_KERNEL, text
    assert "bounded wait" in text
    # a fresh solver of the product library in the same process
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(40, 36, seed=9, bc="symmetric", with_table=True)
    want, want_dts, _ = oracle.run(s, s.state, 4)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        dts = []
        for _ in range(4):
            sol.step()
            dts.append(sol.dt)
        assert np.array_equal(np.array(dts), want_dts)
        assert np.array_equal(sol.get_state(), want)
