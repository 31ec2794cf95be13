"""The discrete adjoint of the CUDA step (rmhd2d_adjoint_forward/backward).

* Against the oracle's tangent (the templated restatement on dual numbers):
  <seed, dU_N/d(direction)> must equal <gradient, direction> -- both are
  exact derivatives of the same frozen-dt map, so to round-off (ADJ_REL).
* Against central finite differences (h = 1e-6) of the CUDA fixed-dt
  forward: FD_REL, the agreement the adjoint is specified to reach.
* The checkpoint interval changes nothing (segments are recomputed bit for
  bit; a kept whole trajectory gives the same gradient with no recompute),
  and backward leaves the solver at the end of the forward run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ADJ_REL = 1e-10
FD_REL = 1e-6


def _dirs(setup, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(setup.state.shape)
    d[..., (1, 2, 3)] *= 1e-2
    d[..., (0, 4, 5, 6, 7)] *= 1e-3
    deta = rng.standard_normal((setup.nx, setup.ny)) * 1e-4
    return d, deta


def _eta_field(setup):
    return setup.eta_table if setup.eta_table is not None else np.full((setup.nx, setup.ny), setup.eta)


def _ghost_gradient_is_zero(gs, nx, bc):
    """Ghost entries of dJ/dU_0 are 0 (set_state's boundary overwrites them),
    except, with symmetric x walls, the lower wall face bY(c, 2) that the x
    walls' normal-B integration reads (c = 3, 4, nx-6, nx-5, nx-4)."""
    ghost = np.ones(gs.shape[:2], bool)
    ghost[3:-3, 3:-3] = False
    mask = np.repeat(ghost[..., None], 8, axis=2)
    if bc == "symmetric":
        for c in (3, 4, nx - 6, nx - 5, nx - 4):
            mask[c, 2, 5] = False
    return np.all(gs[mask] == 0)


@pytest.mark.parametrize("with_table,shape,nsteps,interval,bc,bc_y", [
    (False, (20, 18), 5, 2, "periodic", None),
    (True, (26, 21), 6, 0, "periodic", None),
    (True, (16, 16), 4, 4, "periodic", None),
    (False, (20, 18), 5, 2, "symmetric", None),
    (True, (23, 26), 6, 0, "symmetric", None),
    (True, (18, 21), 4, 2, "periodic", "symmetric"),
    (False, (21, 17), 5, 0, "symmetric", "periodic"),
    (True, (22, 19), 5, -1, "symmetric", None),        # the whole trajectory kept
])
def test_adjoint_matches_oracle_tangent(gpu, oracle, tangent, with_table, shape, nsteps, interval, bc, bc_y):
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(*shape, seed=21, bc=bc, bc_y=bc_y, with_table=with_table)
    ref, ref_dts, crashed = oracle.run(s, s.state, nsteps)
    assert crashed == -1
    w = np.random.default_rng(5).standard_normal(s.state.shape)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.adjoint_forward(nsteps, interval)
        dts = sol.adjoint_dts()
        assert np.array_equal(dts, ref_dts)
        assert np.array_equal(sol.get_state(), ref)
        gs, ge = sol.adjoint_backward(w)
    assert _ghost_gradient_is_zero(gs, s.nx, bc)
    for k in range(3):
        d, deta = _dirs(s, 100 + k)
        _, dU = tangent.tangent(s, s.state, d, dts, deta=deta)
        jvp = float((w * dU).sum())
        vjp_state = float((gs * d).sum())
        vjp_eta = float((ge * deta).sum())
        _, dU_eta = tangent.tangent(s, s.state, np.zeros_like(d), dts, deta=deta)
        assert vjp_eta == pytest.approx(float((w * dU_eta).sum()), rel=ADJ_REL, abs=1e-14)
        assert vjp_state + vjp_eta == pytest.approx(jvp, rel=ADJ_REL, abs=1e-14)


def test_adjoint_full_gradient_on_a_small_grid(gpu, tangent):
    """Every component of dJ/dU_0 and dJ/d eta on a 12x12 interior against
    the oracle's tangent along each unit direction."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(12, 12, seed=8, bc="periodic", with_table=True)
    w = np.random.default_rng(9).standard_normal(s.state.shape)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.adjoint_forward(3, 0)
        dts = sol.adjoint_dts()
        gs, ge = sol.adjoint_backward(w)
    rng = np.random.default_rng(10)
    cells = [(i, j) for i in range(3, s.nx - 3) for j in range(3, s.ny - 3)]
    pick = [cells[t] for t in rng.choice(len(cells), 24, replace=False)]
    for (i, j) in pick:
        for f in range(8):
            d = np.zeros_like(s.state)
            d[i, j, f] = 1.0
            _, dU = tangent.tangent(s, s.state, d, dts)
            want = float((w * dU).sum())
            assert gs[i, j, f] == pytest.approx(want, rel=1e-9, abs=1e-12), (i, j, f)
        de = np.zeros((s.nx, s.ny))
        de[i, j] = 1.0
        _, dU = tangent.tangent(s, s.state, np.zeros_like(s.state), dts, deta=de)
        assert ge[i, j] == pytest.approx(float((w * dU).sum()), rel=1e-9, abs=1e-12), (i, j)


def test_checkpoint_interval_changes_nothing_and_state_is_restored(gpu):
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.orszag_tang(48)
    w = np.random.default_rng(1).standard_normal(s.state.shape)
    grads = []
    for interval in (1, 3, 0, 10, -1):   # -1: the whole trajectory kept, nothing recomputed
        with Solver.from_setup(s, precision="fp64_exact") as sol:
            sol.adjoint_forward(10, interval)
            end = sol.get_state().copy()
            t_end, dt_end = sol.total_time, sol.dt
            g1 = sol.adjoint_backward(w)
            assert np.array_equal(sol.get_state(), end)
            assert sol.total_time == t_end and sol.dt == dt_end
            g2 = sol.adjoint_backward(w)
            assert np.array_equal(g1[0], g2[0]) and np.array_equal(g1[1], g2[1])
            grads.append(g1)
    for g in grads[1:]:
        assert np.array_equal(g[0], grads[0][0]) and np.array_equal(g[1], grads[0][1])


def test_adjoint_against_central_differences(gpu):
    """Misfit of the final (rho, bX, bY, bZ), differentiated through the
    torch.autograd harness, against central differences (h = 1e-6) of the
    CUDA forward with the recorded dts, along localized directions
    (momentum and eta on a 3x3 patch).

    The state is a generic smooth one: where a minmod slope is exactly zero
    (e.g. the uniform density and pressure of the Orszag-Tang start) the
    step map has a kink at the base point itself, central differences then
    converge to the mean of the two one-sided derivatives, and no gradient
    agrees with them.  A limiter kink within h of the base point spoils a
    difference quotient of that h only, so each direction is held to the
    better of h = 1e-6 and 1e-7.  The two misfits are differenced cell by
    cell (misfit_difference), not as two large sums."""
    import torch

    from adjoint_harness import FrozenDtRun, misfit, misfit_difference
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(48, 48, seed=3, bc="periodic", with_table=True)
    nsteps = 10
    eta0 = s.eta_table.copy()
    target = s.state.copy()
    sol = Solver.from_setup(s, precision="fp64_exact")
    try:
        st0 = torch.tensor(s.state, requires_grad=True)
        eta = torch.tensor(eta0, requires_grad=True)
        final = FrozenDtRun.apply(st0, eta, sol, nsteps, 0)
        J = misfit(final, torch.from_numpy(target))
        J.backward()
        dts = sol.adjoint_dts()

        def final_of(state, eta_f):
            sol.set_eta_table(eta_f)
            sol.set_state(state, apply_boundary=True)
            sol.run_fixed_dt(dts)
            return sol.get_state()

        rng = np.random.default_rng(7)
        for _ in range(4):
            d = np.zeros_like(s.state)
            de = np.zeros_like(eta0)
            i0, j0 = rng.integers(3, s.nx - 6), rng.integers(3, s.ny - 6)
            d[i0:i0 + 3, j0:j0 + 3, 1:3] = rng.standard_normal((3, 3, 2))
            de[i0:i0 + 3, j0:j0 + 3] = rng.standard_normal((3, 3)) * eta0[i0:i0 + 3, j0:j0 + 3]
            ad = float((st0.grad.numpy() * d).sum() + (eta.grad.numpy() * de).sum())
            errs = []
            for h in (1e-6, 1e-7):
                fd = misfit_difference(final_of(s.state + h * d, eta0 + h * de),
                                       final_of(s.state - h * d, eta0 - h * de), target) / (2 * h)
                errs.append(abs(fd - ad) / abs(ad))
            assert min(errs) <= FD_REL, (errs, ad)
    finally:
        sol.close()


def test_adjoint_rejects_other_walls(gpu):
    from resistivemhd_gpu_b200 import Solver, _lib, setups

    s = setups.random_smooth_state(20, 18, seed=1, bc="periodic", bc_y="zero_gradient")
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        with pytest.raises(_lib.RMHDError):
            sol.adjoint_forward(2)


def test_adjoint_needs_a_recorded_run(gpu):
    """backward and adjoint_dts are refused before a forward run and after
    adjoint_release, and a refused call leaves the solver stepping with the
    CFL dt."""
    from resistivemhd_gpu_b200 import Solver, _lib, setups

    s = setups.random_smooth_state(20, 18, seed=2, bc="periodic")
    with Solver.from_setup(s, precision="fp64_exact") as sol, \
            Solver.from_setup(s, precision="fp64_exact") as ref:
        seed = np.zeros_like(s.state)
        with pytest.raises(_lib.RMHDError):
            sol.adjoint_backward(seed)
        sol.adjoint_forward(2)
        sol.adjoint_release()
        with pytest.raises(_lib.RMHDError):
            sol.adjoint_backward(seed)
        with pytest.raises(_lib.RMHDError):
            sol.adjoint_dts()
        ref.run(2)
        sol.run(3)
        ref.run(3)
        assert sol.dt == ref.dt
        assert np.array_equal(sol.get_state(), ref.get_state())


def test_adjoint_on_the_harris_sheet(gpu, tangent):
    """Symmetric walls and the eta table of the Harris workload (64 x 32):
    the gradient along seeded directions against the oracle's tangent.

    Here the fast and Alfven waves meet and the HLLD star states' N and D
    are differences of nearly equal terms.  With those recomputed through
    contracted multiply-adds the reverse was 1e-6 off; formed exactly
    rounded, as the forward forms them, it holds ADJ_REL here as everywhere
    (on the CPU build of the same kernels too, tests/test_adjoint_host.py)."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.harris_sheet(64, 32)
    w = np.random.default_rng(3).standard_normal(s.state.shape)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.adjoint_forward(6, 0)
        dts = sol.adjoint_dts()
        gs, ge = sol.adjoint_backward(w)
    assert _ghost_gradient_is_zero(gs, s.nx, "symmetric")
    for k in range(2):
        d, deta = _dirs(s, 200 + k)
        _, dU = tangent.tangent(s, s.state, d, dts, deta=deta)
        assert float((gs * d).sum() + (ge * deta).sum()) == pytest.approx(float((w * dU).sum()), rel=ADJ_REL,
                                                                            abs=1e-14)
