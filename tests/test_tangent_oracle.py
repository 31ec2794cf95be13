"""The templated restatement (oracle/rmhd2d_tangent.cpp) that checks the
discrete adjoint: on doubles it must be the C oracle bit for bit, and on
dual numbers its derivative must agree with central differences of the
fixed-dt step map."""
import numpy as np
import pytest


@pytest.mark.parametrize("bc,bc_y,table,shape", [
    ("periodic", None, False, (17, 23)),
    ("symmetric", None, True, (19, 14)),
    ("periodic", "symmetric", False, (16, 12)),
])
def test_template_on_doubles_is_the_c_oracle(oracle, tangent, bc, bc_y, table, shape):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=5, bc=bc, bc_y=bc_y, with_table=table)
    ref, dts, crashed = oracle.run(s, s.state, 5)
    assert crashed == -1
    out = tangent.run_fixed_dt(s, s.state, dts)
    assert np.array_equal(out, ref)
    # the dual-number instance carries the same values
    val, _ = tangent.tangent(s, s.state, np.zeros_like(s.state), dts)
    assert np.array_equal(val, ref)


def _misfit_dir(setup, seed):
    rng = np.random.default_rng(seed)
    d = np.zeros_like(setup.state)
    d[3:-3, 3:-3, :] = rng.standard_normal(d[3:-3, 3:-3, :].shape)
    d[..., (1, 2)] *= 1e-2
    d[..., (0, 4, 5, 6, 7)] *= 1e-3
    return d


@pytest.mark.parametrize("with_table", [False, True])
def test_tangent_matches_central_differences(oracle, tangent, with_table):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(14, 12, seed=9, bc="periodic", with_table=with_table)
    _, dts, _ = oracle.run(s, s.state, 4)
    d = _misfit_dir(s, 1)
    deta = np.random.default_rng(2).standard_normal((s.nx, s.ny)) * (s.eta * 0.3)
    w = np.random.default_rng(3).standard_normal(s.state.shape)
    _, dU = tangent.tangent(s, s.state, d, dts, deta=deta)
    jvp = float((w * dU).sum())

    def J(h):
        st = s.state + h * d
        if with_table:
            s2 = setups.Setup(s.name, st, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta, s.eta_table + h * deta, s.bc)
        else:
            s2 = setups.Setup(s.name, st, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta,
                              np.full((s.nx, s.ny), s.eta) + h * deta, s.bc)
        return float((w * tangent.run_fixed_dt(s2, st, dts)).sum())

    h = 1e-6
    fd = (J(h) - J(-h)) / (2 * h)
    assert abs(fd - jvp) <= 1e-6 * max(abs(jvp), 1e-12), (fd, jvp)


def test_operation_count_runs_the_same_arithmetic(oracle, tangent):
    """The operation-counting instantiation of the template gives the double
    run's bits, and a count per cell-update of the size the reference's
    algorithm implies (each interface's HLLD with all six candidates)."""
    from resistivemhd_gpu_b200 import setups

    s = setups.orszag_tang(32)
    _, dts, _ = oracle.run(s, s.state, 2)
    ref = tangent.run_fixed_dt(s, s.state, dts)
    out, c = tangent.count_ops(s, s.state, dts)
    assert np.array_equal(out, ref)
    per_cell = (c["add"] + c["mul"] + c["div"] + c["sqrt"]) / (s.interior_cells * len(dts))
    assert 3000 < per_cell < 6000, c
    assert c["div"] > 0 and c["sqrt"] > 0
