"""Parity of the CUDA path (through the C ABI) with the oracle and the
reference's golden outputs.

* FP64 exact variant: bit-identical to the oracle / reference (np.array_equal).
* FP64 fast variant (FMA contraction): relative L1 error per variable
  <= 1e-12 after the stated number of steps, the bar the step must meet
  against the reference.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu

FAST_REL_L1 = 1e-12
# FP32-bulk (single-precision reconstruction and fluxes, FP64 pressure
# recovery, EMF, update and dt): relative L1 <= 1e-5 against FP64.
BULK_REL_L1 = 1e-5


def run_cuda(setup, nsteps, precision="fp64_exact", initial=None, use_run=False):
    from resistivemhd_gpu_b200 import Solver

    with Solver.from_setup(setup, precision=precision, apply_boundary=False) as s:
        s.set_state(setup.state if initial is None else initial, apply_boundary=True)
        dts = []
        if use_run:
            s.run(nsteps)
            dts = None
        else:
            for _ in range(nsteps):
                s.step()
                dts.append(s.dt)
        out = s.get_state()
        total = s.total_time
        crashed = s.check_crashed()
    return out, (np.array(dts) if dts is not None else None), total, crashed


def rel_l1(a, b):
    num = np.abs(a - b).sum(axis=(0, 1))
    den = np.abs(b).sum(axis=(0, 1))
    return num / np.where(den > 0, den, 1.0)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_exact_matches_reference_golden(gpu, name):
    s, init, final, dts, total = load_golden(name)
    out, cdts, ctotal, crashed = run_cuda(s, len(dts), initial=init)
    assert not crashed
    assert np.array_equal(cdts, dts)
    assert np.array_equal(out, final)
    assert ctotal == pytest.approx(total, rel=1e-15)


CASES = [
    ("periodic", False, (33, 70)),   # partial tiles in both directions
    ("periodic", True, (8, 9)),
    ("symmetric", False, (70, 33)),
    ("symmetric", True, (41, 95)),
    ("periodic", False, (6, 6)),     # smallest legal grid
    ("symmetric", False, (6, 31)),
]


@pytest.mark.parametrize("bc,table,shape", CASES)
def test_exact_bitwise_vs_oracle(gpu, oracle, bc, table, shape):
    """Bit-identical states and dt; where the reference crashes (the 6-cell
    wide symmetric box blows up in its first step) the crash is reproduced
    with the same NaN pattern, compared up to the step that crashed."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=5, bc=bc, with_table=table)
    ref, rdts, crashed_at = oracle.run(s, s.state, 7)
    n = 7 if crashed_at < 0 else crashed_at + 1
    out, cdts, _, crashed = run_cuda(s, n)
    assert crashed == (crashed_at >= 0)
    assert np.array_equal(cdts, rdts[:n], equal_nan=True)
    assert np.array_equal(out, ref, equal_nan=True)


@pytest.mark.parametrize("case", ["huge", "nan"])
def test_exact_bitwise_vs_oracle_on_extreme_values(gpu, oracle, case):
    """The exact HLLD forms the selected candidate alone only where all six
    candidates are provably finite (every candidate value below 1e75), and
    the reference's full weighted sum elsewhere.  A patch scaled by 1e80
    (candidate fluxes overflow) and a NaN energy (propagated through the
    weighted sum's 0 * NaN) take the second path; both must still give the
    reference's bits, NaNs included, dt and all (both crash in their first
    step, as the reference does)."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(40, 36, seed=11, bc="periodic")
    st = s.state.copy()
    if case == "huge":
        st[18:21, 15:19, :] *= 1e80
    else:
        st[18, 15, 7] = np.nan
    s.state = st
    ref, rdts, crashed_at = oracle.run(s, st, 3)
    n = 3 if crashed_at < 0 else crashed_at + 1
    out, cdts, _, _ = run_cuda(s, n)
    assert np.array_equal(cdts, rdts[:n], equal_nan=True)
    assert np.array_equal(out, ref, equal_nan=True)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64_fast", "fp32_bulk"])
def test_contracted_variants_propagate_a_nan_energy(gpu, oracle, precision):
    """The contracted variants form an interface with NaN wave speeds after
    their flux loop (the common-case flux declines it) as a NaN flux, as the
    reference's weighted sum does: after one step the same cells are
    non-finite as in the oracle's run, and the crash flag is raised."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(40, 36, seed=11, bc="periodic")
    st = s.state.copy()
    st[18, 15, 7] = np.nan
    s.state = st
    ref, _, crashed_at = oracle.run(s, st, 1)
    out, _, _, crashed = run_cuda(s, 1, precision=precision)
    assert crashed_at == 0 and crashed
    assert np.array_equal(~np.isfinite(out), ~np.isfinite(ref))


@pytest.mark.parametrize("bc,bc_y,table,shape", [
    ("periodic", "symmetric", False, (40, 33)),   # oneStepRK2PeriodicXSymmetricY
    ("periodic", "symmetric", True, (17, 70)),
    ("symmetric", "periodic", False, (35, 38)),
])
def test_mixed_walls_bitwise_vs_oracle(gpu, oracle, bc, bc_y, table, shape):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=8, bc=bc, bc_y=bc_y, with_table=table)
    ref, rdts, crashed_at = oracle.run(s, s.state, 8)
    assert crashed_at == -1
    out, cdts, _, crashed = run_cuda(s, 8)
    assert not crashed
    assert np.array_equal(cdts, rdts)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("bc,table,shape", CASES[:4])
def test_fast_within_tolerance(gpu, oracle, bc, table, shape):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=6, bc=bc, with_table=table)
    ref, _, _ = oracle.run(s, s.state, 10)
    out, _, _, crashed = run_cuda(s, 10, precision="fp64_fast")
    assert not crashed
    assert rel_l1(out, ref).max() <= FAST_REL_L1


@pytest.mark.parametrize("bc,table,shape", CASES[:4])
def test_fp32_bulk_within_tolerance(gpu, oracle, bc, table, shape):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=6, bc=bc, with_table=table)
    ref, _, _ = oracle.run(s, s.state, 10)
    out, _, _, crashed = run_cuda(s, 10, precision="fp32_bulk")
    assert not crashed
    err = rel_l1(out, ref)
    assert err.max() <= BULK_REL_L1
    assert err.max() > 0.0   # it is a different arithmetic, not the FP64 path


def test_fp32_bulk_orszag_tang_and_harris(gpu, oracle):
    from resistivemhd_gpu_b200 import setups

    for s, n in ((setups.orszag_tang(256), 100), (setups.harris_sheet(256, 128), 40)):
        ref, _, _ = oracle.run(s, s.state, n)
        out, _, _, crashed = run_cuda(s, n, precision="fp32_bulk")
        assert not crashed
        assert rel_l1(out, ref).max() <= BULK_REL_L1, s.name


def test_run_graph_equals_step_loop(gpu):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(40, 36, seed=9, bc="symmetric", with_table=True)
    a, _, ta, _ = run_cuda(s, 7)
    b, _, tb, _ = run_cuda(s, 7, use_run=True)
    assert np.array_equal(a, b)
    assert ta == tb


def test_calculate_dt_matches_oracle(gpu, oracle):
    from resistivemhd_gpu_b200 import Solver, setups

    for bc in ("periodic", "symmetric"):
        s = setups.random_smooth_state(30, 20, seed=3, bc=bc)
        st = oracle.boundary(s, s.state)
        with Solver.from_setup(s, apply_boundary=True) as sol:
            assert sol.calculate_dt() == oracle.calc_dt(s, st)


def test_orszag_tang_256_100_steps(gpu, oracle):
    """The reference's CPU-runnable config: OT 256^2, 100 steps."""
    from resistivemhd_gpu_b200 import setups

    s = setups.orszag_tang(256)
    ref, rdts, _ = oracle.run(s, s.state, 100)
    out, cdts, _, _ = run_cuda(s, 100)
    assert np.array_equal(cdts, rdts)
    assert np.array_equal(out, ref)
    fast, _, _, _ = run_cuda(s, 100, precision="fp64_fast")
    assert rel_l1(fast, ref).max() <= FAST_REL_L1
    bx, by = out[..., 4], out[..., 5]
    div = (bx[3:-3, 3:-3] - bx[2:-4, 3:-3]) / s.dx + (by[3:-3, 3:-3] - by[3:-3, 2:-4]) / s.dy
    assert np.abs(div).max() < 1e-10


def test_harris_symmetric_eta_table(gpu, oracle):
    from resistivemhd_gpu_b200 import setups

    s = setups.harris_sheet(256, 128)
    ref, rdts, _ = oracle.run(s, s.state, 20)
    out, cdts, _, _ = run_cuda(s, 20)
    assert np.array_equal(cdts, rdts)
    assert np.array_equal(out, ref)


def test_save_load_resume(gpu, tmp_path):
    from resistivemhd_gpu_b200 import Solver, read_snapshot, setups

    s = setups.random_smooth_state(30, 26, seed=4, bc="symmetric")
    with Solver.from_setup(s) as a:
        a.run(4)
        path = a.save(str(tmp_path), "snap", 4)
        snap = read_snapshot(path, s.nx, s.ny)
        assert np.array_equal(snap, a.get_state())
        a.run(3)
        ref = a.get_state()
    with Solver.from_setup(s) as b:
        b.load(path)
        b.run(3)
        assert np.array_equal(b.get_state(), ref)


def test_crash_flag_on_host_injected_nan(gpu):
    """A NaN energy injected into the host state before upload is reported by
    check_crashed after the next step (no GPU fault involved)."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(20, 20, seed=2)
    st = s.state.copy()
    st[10, 10, 7] = np.nan
    with Solver.from_setup(s, apply_boundary=False) as sol:
        sol.set_state(st, apply_boundary=True)
        assert sol.check_crashed()
        sol.step()
        assert sol.check_crashed()
    with Solver.from_setup(s) as sol:
        sol.step()
        assert not sol.check_crashed()


def test_reference_class_mirror(gpu, oracle):
    from resistivemhd_gpu_b200 import ResistiveMHD2D, setups

    s = setups.orszag_tang(40)

    class OT(ResistiveMHD2D):
        def initializeU(self):
            self.U[...] = s.state

    sim = OT(s.nx, s.ny, s.dx, s.dy, gamma_mhd=s.gamma, CFL=s.cfl, EPS=s.eps, eta=s.eta)
    sim.initialize()
    total = 0.0
    for _ in range(5):
        sim.oneStepRK2()
        assert not sim.checkCalculationIsCrashed()
        total += sim.dt
    ref, rdts, _ = oracle.run(s, s.state, 5)
    assert np.array_equal(sim.getU(), ref)
    assert sim.totalTime == total


@pytest.mark.skipif(os.environ.get("RMHD_SKIP_LARGE") == "1", reason="large-grid property test disabled")
def test_full_size_properties(gpu):
    """Harris 2048x1024 (the benchmark size): no crash, div B at round-off;
    periodic 1024^2 OT: interior sums of rho and e conserved to round-off."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.harris_sheet(2048, 1024)
    with Solver.from_setup(s, precision="fp64_fast") as sol:
        sol.run(20)
        assert not sol.check_crashed()
        u = sol.get_state()
    bx, by = u[..., 4], u[..., 5]
    div = (bx[3:-3, 3:-3] - bx[2:-4, 3:-3]) / s.dx + (by[3:-3, 3:-3] - by[3:-3, 2:-4]) / s.dy
    assert np.abs(div).max() < 1e-9
    o = setups.orszag_tang(1024)
    with Solver.from_setup(o, precision="fp64_fast") as sol:
        u0 = sol.get_state()
        sol.run(20)
        u1 = sol.get_state()
    for f in (0, 7):
        a0, a1 = u0[3:-3, 3:-3, f].sum(), u1[3:-3, 3:-3, f].sum()
        assert abs(a1 - a0) <= 1e-11 * abs(a0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp32_bulk", "fp64_fast"])
def test_orszag_tang_past_the_degenerate_fast_speed(gpu, precision):
    """Orszag-Tang keeps bZ = 0 and lets bY cross zero, so the fast-speed
    discriminant (cs2 + ca2)^2 - 4 cs2 va2 reaches 0 where cs ~ ca; formed
    with cancellation it rounded below zero in single precision and the
    FP32-bulk run crashed near t = 2.  The run must stay finite and follow
    the FP64 run."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.ot_adjoint(256)
    with Solver.from_setup(s, precision="fp64_exact") as ref:
        ref.run(1100)
        assert not ref.check_crashed()
        want, t_want = ref.get_state(), ref.total_time
    with Solver.from_setup(s, precision=precision) as sol:
        sol.run(1100)
        assert not sol.check_crashed()
        got = sol.get_state()
        assert sol.total_time == pytest.approx(t_want, rel=1e-6)
    rho = np.abs(got[3:-3, 3:-3, 0] - want[3:-3, 3:-3, 0]).sum() / np.abs(want[3:-3, 3:-3, 0]).sum()
    assert rho < (1e-4 if precision == "fp32_bulk" else 1e-9)


@pytest.mark.gpu
def test_fp32_bulk_harris_past_the_degenerate_star_denominator(gpu):
    """On the 2048 x 1024 Harris sheet the HLLD star denominator
    rho (S - u)(S - SM) - bX^2 of some x-faces falls below what single
    precision resolves (bX ~ 1, |bY| ~ 4e-5 at about step 130); dividing by
    its rounding residue crashed the FP32-bulk run.  The run must stay
    finite and follow the FP64 run at the same time steps."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.harris_sheet(2048, 1024)
    nsteps = 200
    with Solver.from_setup(s, precision="fp64_fast") as ref:
        dts = []
        for _ in range(nsteps):
            ref.step()
            dts.append(ref.dt)
        assert not ref.check_crashed()
        want = ref.get_state()
    with Solver.from_setup(s, precision="fp32_bulk") as sol:
        sol.run(nsteps)
        assert not sol.check_crashed()
        got = sol.get_state()
        assert sol.total_time == pytest.approx(sum(dts), rel=1e-6)
    err = rel_l1(got[3:-3, 3:-3], want[3:-3, 3:-3])
    assert np.all(err[[0, 4, 5, 7]] < BULK_REL_L1), err
