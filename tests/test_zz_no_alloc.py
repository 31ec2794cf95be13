"""rmhd2d_calculate_dt_noalloc (the allocation-free CFL dt of a state held in
the caller's device memory) against rmhd2d_calculate_dt of a solver holding
the same state.  The file name makes pytest collect it last, so it runs
after every other test of a session as well as alone.

Both entry points evaluate the same FP64 rate without fused multiply-add,
so equal values are expected; REL_TOL is the bound the test holds them to."""
import ctypes

import numpy as np
import pytest

REL_TOL = 1e-14


def _config(setup, device=0):
    from resistivemhd_gpu_b200 import Solver

    return Solver.make_config(setup.nx, setup.ny, setup.dx, setup.dy, gamma=setup.gamma, cfl=setup.cfl,
                              eps=setup.eps, eta=setup.eta, bc=setup.bc, bc_y=setup.bc_y, device=device)


def _noalloc_dt(setup, device_state) -> float:
    """device_state: a CUDA tensor the caller (this test) allocated."""
    import torch
    from resistivemhd_gpu_b200 import _lib

    torch.cuda.synchronize()
    cfg = _config(setup)
    out = ctypes.c_double(float("nan"))
    _lib.check(_lib.load().rmhd2d_calculate_dt_noalloc(ctypes.byref(cfg), ctypes.c_void_p(device_state.data_ptr()),
                                                       ctypes.byref(out)), None)
    return out.value


def _solver_dt_and_state(setup, nsteps):
    from resistivemhd_gpu_b200 import Solver

    with Solver.from_setup(setup, precision="fp64_exact") as s:
        s.run(nsteps)
        return s.calculate_dt(), s.get_state()


def _close(a, b):
    return a == b or abs(a - b) <= REL_TOL * abs(b)


@pytest.mark.gpu
def test_noalloc_dt_matches_solver_two_calls_in_a_row(gpu):
    import torch
    from resistivemhd_gpu_b200 import setups

    cases = [(setups.harris_sheet(256, 128), 3), (setups.orszag_tang(64), 2)]
    expected, states = [], []
    for setup, nsteps in cases:
        dt, state = _solver_dt_and_state(setup, nsteps)
        expected.append(dt)
        states.append(torch.from_numpy(np.ascontiguousarray(state)).to("cuda:0"))
    assert expected[0] != expected[1], "the two cases must differ for the second call to prove anything"
    got = [_noalloc_dt(setup, st) for (setup, _), st in zip(cases, states)]
    for g, e in zip(got, expected):
        assert np.isfinite(g) and _close(g, e), (g, e)
    # and once more in the opposite order, through the same scratch
    again = [_noalloc_dt(cases[1][0], states[1]), _noalloc_dt(cases[0][0], states[0])]
    assert _close(again[0], expected[1]) and _close(again[1], expected[0])


@pytest.mark.gpu
def test_noalloc_dt_nan_semantics_match_solver(gpu):
    """The reference's min_element skips a NaN candidate except in cell 0,
    where the NaN minimum then loses to the diffusive limit in fmin."""
    import torch
    from resistivemhd_gpu_b200 import Solver, setups

    setup = setups.random_smooth_state(40, 36, seed=7, bc="periodic")
    for cell in [(0, 0), (17, 11)]:
        st = setup.state.copy()
        st[cell][7] = np.nan
        with Solver.from_setup(setup, precision="fp64_exact", apply_boundary=False) as s:
            s.set_state(st, apply_boundary=False)
            want = s.calculate_dt()
        got = _noalloc_dt(setup, torch.from_numpy(np.ascontiguousarray(st)).to("cuda:0"))
        assert np.isfinite(want) and _close(got, want), (cell, got, want)
        if cell == (0, 0):
            assert setup.eta > 0
            assert want == min(setup.dx * setup.dx / setup.eta, setup.dy * setup.dy / setup.eta) * setup.cfl


def test_noalloc_dt_rejects_grids_above_the_scratch_limit():
    """Rejected before any CUDA call, so this runs without a GPU."""
    from resistivemhd_gpu_b200 import _lib, setups

    lib = _lib.load()
    setup = setups.random_smooth_state(12, 12, seed=1)
    cfg = _config(setup)
    cfg.nx, cfg.ny = 4097, 4096
    host = np.zeros(8, dtype=np.float64)
    out = ctypes.c_double(-1.0)
    st = lib.rmhd2d_calculate_dt_noalloc(ctypes.byref(cfg), ctypes.c_void_p(host.ctypes.data), ctypes.byref(out))
    assert st == 1  # RMHD2D_ERR_INVALID
    assert "RMHD2D_NOALLOC_MAX_CELLS" in lib.rmhd2d_last_error(None).decode()
    assert out.value == -1.0
