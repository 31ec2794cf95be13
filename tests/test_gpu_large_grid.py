"""Solvers created one after another on grids of more than 2^24 cells.

rmhd2d_create clears the new state planes.  Issued on the legacy default
stream, which the solver's non-blocking stream does not wait for, those
clears could still be running when set_state's host-to-device copy landed
and zeroed its first chunk (rows i = 0..7 of every field of an 8192 x 2048
grid); the CFL dt then fell back to the diffusive limit and the first step
blew up.  The clears are now ordered on the solver's stream."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_consecutive_solvers_keep_the_uploaded_state(gpu, oracle):
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.plasmoid_sheet(8192, 2048)
    want_dt = oracle.calc_dt(s, s.state)
    for _ in range(3):
        with Solver.from_setup(s, precision="fp64_exact", apply_boundary=False) as sol:
            dt = sol.calculate_dt()
            got = sol.get_state()
        assert np.array_equal(got, s.state)
        assert dt == want_dt


def test_plasmoid_first_steps_match_the_oracle(gpu, oracle):
    """Two steps of the 8192 x 2048 thin sheet, bit for bit, after another
    solver of that size was created and destroyed."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.plasmoid_sheet(8192, 2048)
    with Solver.from_setup(s, precision="fp64_fast") as other:
        other.step()
    want, dts, crashed_at = oracle.run(s, s.state, 2)
    assert crashed_at == -1
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        got_dts = []
        for _ in range(2):
            sol.step()
            got_dts.append(sol.dt)
        got = sol.get_state()
    assert got_dts == list(dts)
    assert np.array_equal(got, want)
