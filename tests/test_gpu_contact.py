"""The CT-Contact step (cfg.ct_scheme = RMHD2D_CT_CONTACT) against the
oracle's orc_step_contact: states and per-step dt bit for bit, stepping one
call at a time and replayed from graphs, on periodic, symmetric, mixed walls
and with an eta table.  The multi-GPU library the EMF comes from needs MPI
and is not built here, so the oracle restates its ct.cu arithmetic; the
fluxes, boundaries and CT update it shares with the other step are pinned to
the reference."""
import dataclasses

import numpy as np
import pytest

CASES = [
    ("ot", lambda s: s.orszag_tang(48)),
    ("smooth_table", lambda s: s.random_smooth_state(30, 26, seed=3, bc="periodic", with_table=True)),
    ("harris", lambda s: s.harris_sheet(64, 32)),
    ("mixed", lambda s: s.random_smooth_state(20, 18, seed=5, bc="periodic", bc_y="symmetric")),
    ("ragged_symmetric", lambda s: s.random_smooth_state(13, 21, seed=6, bc="symmetric", with_table=True)),
]


def test_contact_step_invariants_on_the_oracle(oracle):
    """CT keeps the discrete div B of the start; the periodic walls keep
    sum(rho) and sum(e); the EMF differs from the stage-1 one."""
    from resistivemhd_gpu_b200 import setups

    s = setups.orszag_tang(48)
    sc = dataclasses.replace(s, ct="contact")
    out, dts, crashed = oracle.run(sc, s.state, 20)
    assert crashed == -1 and np.isfinite(out).all()
    bx, by = out[..., 4], out[..., 5]
    div = (bx[3:-3, 3:-3] - bx[2:-4, 3:-3]) / s.dx + (by[3:-3, 3:-3] - by[3:-3, 2:-4]) / s.dy
    assert np.abs(div).max() < 1e-12
    init = oracle.boundary(s, s.state)
    for f in (0, 7):
        assert abs(out[3:-3, 3:-3, f].sum() - init[3:-3, 3:-3, f].sum()) <= 1e-12 * abs(init[3:-3, 3:-3, f].sum())
    ref, _, _ = oracle.run(s, s.state, 20)
    assert not np.array_equal(out, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name,make", CASES)
def test_contact_step_matches_oracle_bit_for_bit(gpu, oracle, name, make):
    from resistivemhd_gpu_b200 import Solver, setups

    s = dataclasses.replace(make(setups), ct="contact")
    n = 8
    ref, rdts, crashed = oracle.run(s, s.state, n)
    assert crashed == -1
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        dts = []
        for _ in range(n):
            sol.step()
            dts.append(sol.dt)
        assert np.array_equal(np.array(dts), rdts)
        assert np.array_equal(sol.get_state(), ref)
        assert sol.calculate_dt() == oracle.calc_dt(s, ref)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.run(n)                                   # graph replay
        assert np.array_equal(sol.get_state(), ref)
        assert sol.total_time == pytest.approx(rdts.sum(), rel=1e-15)


@pytest.mark.gpu
def test_contact_runs_long_and_conserves(gpu):
    from resistivemhd_gpu_b200 import Solver, setups

    s = dataclasses.replace(setups.orszag_tang(128), ct="contact")
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        start = sol.get_state()
        sol.run(400)
        assert not sol.check_crashed()
        out = sol.get_state()
    bx, by = out[..., 4], out[..., 5]
    div = (bx[3:-3, 3:-3] - bx[2:-4, 3:-3]) / s.dx + (by[3:-3, 3:-3] - by[3:-3, 2:-4]) / s.dy
    assert np.abs(div).max() < 1e-11
    for f in (0, 7):
        assert abs(out[3:-3, 3:-3, f].sum() - start[3:-3, 3:-3, f].sum()) <= 1e-11 * abs(start[3:-3, 3:-3, f].sum())


@pytest.mark.gpu
def test_contact_refuses_batch_adjoint_and_profile(gpu):
    from resistivemhd_gpu_b200 import Batch, Solver, _lib, setups

    s = dataclasses.replace(setups.orszag_tang(32), ct="contact")
    with Solver.from_setup(s) as sol:
        with pytest.raises(_lib.RMHDError):
            sol.adjoint_forward(2)
        with pytest.raises(_lib.RMHDError):
            sol.profile_step()
    with pytest.raises(_lib.RMHDError):
        Batch([s, s])


@pytest.mark.gpu
@pytest.mark.parametrize("ct", ["stage1", "contact"])
def test_fixed_dt_replay_equals_the_run(gpu, ct):
    """A run replayed with its own recorded dts (rmhd2d_run_fixed_dt) gives
    the run's states bit for bit, with either CT scheme: the stage kernels
    read each step's dt from the replay's table, CT-Contact's pipeline from
    the control block."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = dataclasses.replace(setups.harris_sheet(64, 32), ct=ct)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        dts = []
        for _ in range(5):
            sol.step()
            dts.append(sol.dt)
        want = sol.get_state()
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.run_fixed_dt(dts)
        got = sol.get_state()
        assert sol.dt == dts[-1]
    assert np.array_equal(got, want)
