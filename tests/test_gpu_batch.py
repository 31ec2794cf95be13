"""Tile shapes and batches of independent runs.

The tile decomposition changes no arithmetic: every interface flux and cell
update is computed by the same expressions whatever tile or launch holds it.
The FP64-exact variant (no contraction) is therefore equal bit for bit in a
batch, on the other tile shape and in the single run.  The FP64-fast and
FP32-bulk variants are compiled with fused multiply-add contraction left to
the compiler, which may contract the same source differently in the
persistent batch kernel than in the single-run kernel.  Their batches are
held to FAST_BATCH_REL_L1 and BULK_BATCH_REL_L1 of the single run per
field.  The FP64 bound is rounding level for the fluxes (~1e-16 of O(1)
values) measured against fields as small as the Harris sheet's momenta
(~1e-4 of its energy), i.e. up to ~1e-12 of such a field; the FP32-bulk
bound is 100 times inside that variant's own 1e-5 against FP64."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECISIONS = ["fp64_exact", "fp64_fast", "fp32_bulk"]
FAST_BATCH_REL_L1 = 1e-10
BULK_BATCH_REL_L1 = 1e-7
BATCH_REL_L1 = {"fp64_exact": 0.0, "fp64_fast": FAST_BATCH_REL_L1, "fp32_bulk": BULK_BATCH_REL_L1}


def assert_same(got, ref, precision, what):
    if precision == "fp64_exact":
        assert np.array_equal(got, ref), what
        return
    for f in range(8):
        den = np.abs(ref[..., f]).sum()
        err = np.abs(got[..., f] - ref[..., f]).sum() / max(den, 1e-300)
        assert err <= BATCH_REL_L1[precision], f"{what} field {f}: rel L1 {err:.3e}"


def single(setup, nsteps, precision, shape=0):
    from resistivemhd_gpu_b200 import Solver

    with Solver.from_setup(setup, precision=precision) as s:
        if isinstance(shape, tuple):
            s.set_stage_shapes(*shape)        # (stage 1, stage 2)
        else:
            s.set_tile_shape(shape)
        dts = []
        for _ in range(nsteps):
            s.step()
            dts.append(s.dt)
        return s.get_state(), np.array(dts), s.total_time


def mixed_setups():
    from resistivemhd_gpu_b200 import setups

    return [
        setups.random_smooth_state(40, 36, seed=1, bc="periodic"),
        setups.random_smooth_state(23, 70, seed=2, bc="symmetric", with_table=True),
        setups.orszag_tang(48),
        setups.random_smooth_state(64, 17, seed=3, bc="periodic", bc_y="symmetric", eta=5e-3),
        setups.harris_sheet(96, 48),
    ]


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("shape", [1, 2, 3, 4, 5, (1, 0), (2, 1), (3, 4), (4, 3), (5, 4), (0, 5)])
def test_tile_shapes_equal_shape_0(gpu, precision, shape):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(45, 39, seed=4, bc="symmetric", with_table=True)
    a, da, _ = single(s, 6, precision, shape=0)
    b, db, _ = single(s, 6, precision, shape=shape)
    rel = {"fp64_exact": 0.0, "fp64_fast": 1e-12, "fp32_bulk": 1e-6}[precision]
    assert db == pytest.approx(da, rel=rel, abs=0)
    assert_same(b, a, precision, f"shape {shape}")


@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("launch", [(0, 2), (1, 1), (2, 1), (3, 1), (4, 3)])
def test_batch_equals_single_runs(gpu, precision, launch):
    from resistivemhd_gpu_b200 import Batch

    sets = mixed_setups()
    refs = [single(s, 5, precision) for s in sets]
    with Batch(sets, precision=precision) as b:
        b.set_launch(*launch)
        b.run(5)
        for r, (ref, dts, total) in enumerate(refs):
            m = b[r]
            assert_same(m.get_state(), ref, precision, f"run {r}")
            rel = {"fp64_exact": 0.0, "fp64_fast": 1e-12, "fp32_bulk": 1e-6}[precision]
            assert m.dt == pytest.approx(dts[-1], rel=rel, abs=0)
            assert m.total_time == pytest.approx(total, rel=max(rel, 1e-15))
            assert not m.check_crashed()


def test_batch_odd_steps_and_graph_replay(gpu):
    """Graph replays of 2 steps plus a single step keep every run in step."""
    from resistivemhd_gpu_b200 import Batch

    sets = mixed_setups()[:3]
    refs = [single(s, 7, "fp64_exact") for s in sets]
    with Batch(sets, precision="fp64_exact") as b:
        b.run(3)
        b.run(4)
        for r, (ref, _, _) in enumerate(refs):
            assert np.array_equal(b[r].get_state(), ref)


def test_batch_autotune_restores_state(gpu):
    from resistivemhd_gpu_b200 import Batch

    sets = mixed_setups()
    with Batch(sets, precision="fp64_fast") as b:
        before = [b[r].get_state().copy() for r in range(len(b))]
        shape, ctas = b.autotune(trial_steps=2)
        assert shape in range(6) and ctas in (1, 2, 3)
        table = b.tuning()
        assert [(sh, c) for sh, c, _ in table] == [(0, 1), (0, 2), (1, 1), (1, 2), (2, 1), (3, 1), (4, 1), (4, 2),
                                                   (4, 3), (5, 1), (5, 2), (5, 3)]
        assert all(m > 0 for _, _, m in table)
        assert b.launch == (shape, ctas)
        for r in range(len(b)):
            assert np.array_equal(b[r].get_state(), before[r])
        b.run(3)
    refs = [single(s, 3, "fp64_fast") for s in sets]
    with Batch(sets, precision="fp64_fast") as b:
        b.set_launch(shape, ctas)
        b.run(3)
        for r, (ref, _, _) in enumerate(refs):
            assert_same(b[r].get_state(), ref, "fp64_fast", f"run {r}")


def test_member_cannot_step_alone(gpu):
    from resistivemhd_gpu_b200 import Batch, _lib

    with Batch(mixed_setups()[:2]) as b:
        with pytest.raises(_lib.RMHDError) as e:
            b[0].step()
        assert e.value.status == 4


def test_solver_autotune(gpu):
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.harris_sheet(256, 128)
    with Solver.from_setup(s, precision="fp64_fast") as sol:
        before = sol.get_state().copy()
        shape = sol.autotune(trial_steps=2)
        assert shape in range(6) and sol.tile_shape == shape
        t = sol.tuning()
        assert sorted(t) == [0, 1, 2, 3, 4, 5] and all(a > 0 and b > 0 for a, b in t.values())
        s1, s2 = sol.stage_shapes
        assert s1 == shape and t[s2][1] == min(b for _, b in t.values())
        assert np.array_equal(sol.get_state(), before)
