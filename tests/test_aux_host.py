"""The ghost fill, the CFL reduction and the allocation-free dt on the CPU:
aux_kernels.cu and noalloc_dt.cu compiled for the host (tests/host_build.py;
the kernels that reduce with warp shuffles and atomics run one host thread
per CUDA thread) and driven as the C ABI drives them (tests/aux_host.cpp).
Built without contraction, as nvcc builds them (-fmad=false), the filled
states and the dts must equal the oracle's bit for bit, as
tests/test_walls.py and tests/test_zz_no_alloc.py require of the CUDA runs."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from host_build import compile_unit, link, shim_dir

HERE = Path(__file__).resolve().parent
BC = {"periodic": 0, "symmetric": 1, "zero_gradient": 2, "wall": 3, "flare": 4}
D = ctypes.POINTER(ctypes.c_double)


def build_aux(d: Path, extra: tuple[str, ...] = ()):
    """aux_kernels.cu, noalloc_dt.cu and their drivers as a host library;
    `extra` adds compiler flags to every unit (e.g. sanitizers)."""
    shim_dir(d)
    objs = [compile_unit(d, "aux_kernels.cu", ["-ffp-contract=off", *extra],
                         threaded=("kernel", "rate_kernel", "boundary_batch_kernel")),
            compile_unit(d, "noalloc_dt.cu", ["-ffp-contract=off", *extra], threaded=("dt_noalloc_kernel",))]
    lib = link(d, objs, [HERE / "aux_host.cpp"], "libauxhost.so", extra)
    lib.host_set_state_dt.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 + [
        ctypes.c_int, ctypes.c_int, D, D, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
        ctypes.POINTER(ctypes.c_ulonglong)]
    lib.host_dt_noalloc.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 + [D, D]
    return lib


@pytest.fixture(scope="module")
def aux(tmp_path_factory):
    return build_aux(tmp_path_factory.mktemp("auxhost"))


def set_state_dt(lib, s, state, ghost_rates=False):
    out = np.ascontiguousarray(state, dtype=np.float64).copy()
    dt, crashed, gmax = ctypes.c_double(), ctypes.c_int(), ctypes.c_ulonglong()
    rc = lib.host_set_state_dt(s.nx, s.ny, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta, BC[s.bc],
                               BC[s.bc_y] if s.bc_y else -1, out.ctypes.data_as(D), ctypes.byref(dt),
                               ctypes.byref(crashed), int(ghost_rates), ctypes.byref(gmax))
    assert rc == 0
    return out, dt.value, crashed.value, gmax.value


def dt_noalloc(lib, s, state):
    a = np.ascontiguousarray(state, dtype=np.float64)
    dt = ctypes.c_double()
    assert lib.host_dt_noalloc(s.nx, s.ny, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta, a.ctypes.data_as(D),
                               ctypes.byref(dt)) == 0
    return dt.value


def same(a, b):
    return a == b or (a != a and b != b)


@pytest.mark.parametrize("bcx", ["periodic", "symmetric", "zero_gradient", "flare"])
@pytest.mark.parametrize("bcy", ["periodic", "symmetric", "zero_gradient", "wall"])
def test_ghost_fill_and_dt_equal_oracle(aux, oracle, bcx, bcy):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(17, 14, seed=5, bc=bcx, bc_y=bcy)
    want = oracle.boundary(s, s.state)
    got, dt, crashed, gmax = set_state_dt(aux, s, s.state, ghost_rates=True)
    assert np.array_equal(got, want, equal_nan=True)
    assert same(dt, oracle.calc_dt(s, want))
    assert same(dt_noalloc(aux, s, want), dt)
    assert crashed == 0 and gmax > 0


@pytest.mark.parametrize("bc", ["periodic", "symmetric"])
def test_nan_energy_and_nan_rates(aux, oracle, bc):
    """A NaN energy raises the crash flag; NaN rates are skipped by the
    minimum unless they fall on cell 0, where the reference's min_element
    returns them (the dt is then NaN), for the solver's reduction and the
    allocation-free one alike."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(15, 13, seed=6, bc=bc)
    for cells in ([(7, 6)], [(3, 3), (s.nx - 4, s.ny - 4)], [(s.nx - 6, s.ny - 6)]):
        st = s.state.copy()
        for (i, j) in cells:
            st[i, j, 7] = np.nan
        want = oracle.boundary(s, st)
        got, dt, crashed, _ = set_state_dt(aux, s, st)
        assert np.array_equal(got, want, equal_nan=True)
        assert crashed == 1
        assert same(dt, oracle.calc_dt(s, want))
        assert same(dt_noalloc(aux, s, want), dt)
