"""The CT-Contact step's kernels on the CPU: contact.cu compiled for the host
(tests/host_build.py; the tiled flux kernel, which stages its tile in shared
memory and synchronises the block, runs one host thread per CUDA thread) and
driven as rmhd2d_step_rk2 drives it (tests/contact_host.cpp).  Built without
contraction, as nvcc builds contact.cu (-fmad=false), the states and dts
must equal the oracle's orc_step_contact bit for bit, as
tests/test_gpu_contact.py requires of the CUDA run."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

from host_build import ORACLE, compile_unit, link, shim_dir

HERE = Path(__file__).resolve().parent
BC = {"periodic": 0, "symmetric": 1, "zero_gradient": 2, "wall": 3, "flare": 4}


def build_contact(d: Path, extra: tuple[str, ...] = ()):
    """contact.cu, the oracle and the step driver as a host library; `extra`
    adds compiler flags to every unit (e.g. sanitizers)."""
    shim_dir(d)
    objs = [compile_unit(d, "contact.cu", ["-ffp-contract=off", "-DRMHD_HOST_EMULATION", *extra],
                          threaded=("contact_flux_tiled_kernel",))]
    orc = d / "oracle.o"
    subprocess.run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", *extra, "-fPIC", "-c",
                    str(ORACLE / "rmhd2d_oracle.c"), "-o", str(orc)], check=True, capture_output=True)
    objs.append(str(orc))
    lib = link(d, objs, [HERE / "contact_host.cpp"], "libcontacthost.so", extra)
    D = ctypes.POINTER(ctypes.c_double)
    lib.host_contact_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, D,
                                     D, ctypes.c_int, D]
    lib.host_contact_run.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="module")
def host_contact(tmp_path_factory):
    return build_contact(tmp_path_factory.mktemp("contacthost"))


def run_host(lib, s, nsteps):
    D = ctypes.POINTER(ctypes.c_double)
    tab = None if s.eta_table is None else np.ascontiguousarray(s.eta_table, dtype=np.float64)
    state = np.ascontiguousarray(s.state, dtype=np.float64).copy()
    dts = np.zeros(max(nsteps, 1))
    rc = lib.host_contact_run(s.nx, s.ny, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta, BC[s.bc],
                              BC[s.bc_y] if s.bc_y else -1, None if tab is None else tab.ctypes.data_as(D),
                              state.ctypes.data_as(D), nsteps, dts.ctypes.data_as(D))
    return state, dts[:nsteps], rc - 1 if rc > 0 else -1


@pytest.mark.parametrize("shape,nsteps,bc,bc_y,with_table", [
    ((20, 18), 4, "periodic", None, False),
    ((37, 29), 3, "periodic", None, True),
    ((26, 40), 3, "symmetric", None, True),
    ((23, 19), 3, "periodic", "symmetric", False),
    ((21, 25), 3, "flare", "wall", True),
    ((18, 17), 3, "zero_gradient", "periodic", False),
])
def test_host_contact_step_equals_oracle(host_contact, oracle, shape, nsteps, bc, bc_y, with_table):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=13, bc=bc, bc_y=bc_y, with_table=with_table)
    s.ct = "contact"
    want, want_dts, want_crash = oracle.run(s, s.state, nsteps)
    got, got_dts, got_crash = run_host(host_contact, s, nsteps)
    assert got_crash == want_crash
    assert np.array_equal(got_dts, want_dts)
    assert np.array_equal(got, want, equal_nan=True)
