"""The oracle (C restatement of the reference step) pinned against the
reference's own outputs: the committed golden fixtures (generated by running
the reference library built for the host) and, when oracle/_ref is built,
live runs of the reference."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, load_golden


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_golden_bit_exact(oracle, name):
    s, init, final, dts, total_time = load_golden(name)
    out, odts, crashed = oracle.run(s, init, len(dts))
    assert crashed == -1
    assert np.isfinite(out).all(), "a value the reference never reads reached the state"
    assert np.array_equal(odts, dts)
    assert np.array_equal(out, final)
    assert np.isclose(odts.sum(), total_time, rtol=0, atol=1e-15 * max(1.0, total_time))


def _ref_available(kind="cpu"):
    from oracle.oracle import reference_binary

    return reference_binary(kind, "periodic").exists() and reference_binary(kind, "symmetric").exists()


@pytest.mark.skipif(not _ref_available(), reason="reference host build (oracle/build_ref.py) not present")
@pytest.mark.parametrize("bc,table,shape", [
    ("periodic", False, (17, 23)),     # ragged, odd sizes
    ("symmetric", False, (30, 13)),
    ("symmetric", True, (19, 29)),
    ("periodic", True, (6, 40)),       # thinnest legal interior in x
])
def test_oracle_matches_live_reference(oracle, bc, table, shape):
    from oracle.oracle import run_reference
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=11, bc=bc, with_table=table)
    a, adts, _ = oracle.run(s, s.state, 6)
    b, bdts, info = run_reference(s, s.state, 6, kind="cpu", threads=2)
    assert info["crashed_at"] == -1
    assert np.array_equal(adts, bdts)
    assert np.array_equal(a, b)


def test_oracle_boundary_periodic_is_pure_copy(oracle):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(10, 12, bc="periodic")
    u = oracle.boundary(s, s.state)
    nx, ny = s.nx, s.ny
    inner = u[3:nx - 3, 3:ny - 3]
    tiled = np.tile(inner, (3, 3, 1))
    px, py = nx - 6, ny - 6
    assert np.array_equal(u, tiled[px - 3:px - 3 + nx, py - 3:py - 3 + ny])


def test_oracle_divergence_free_and_conservative(oracle):
    """Invariants the reference's CT and flux-difference update give: the
    discrete div B stays at round-off and, with periodic walls, the interior
    sums of rho and e change only by round-off."""
    from resistivemhd_gpu_b200 import setups

    s = setups.orszag_tang(48)
    out, _, _ = oracle.run(s, s.state, 30)
    bx, by = out[..., 4], out[..., 5]
    div = (bx[3:-3, 3:-3] - bx[2:-4, 3:-3]) / s.dx + (by[3:-3, 3:-3] - by[3:-3, 2:-4]) / s.dy
    assert np.abs(div).max() < 1e-11
    init = oracle.boundary(s, s.state)
    for f in (0, 7):
        a0 = init[3:-3, 3:-3, f].sum()
        a1 = out[3:-3, 3:-3, f].sum()
        assert abs(a1 - a0) <= 1e-11 * abs(a0)


def test_oracle_crash_flag_on_host_injected_nan(oracle):
    """Failure detection is exercised by a fault injected on the host: a NaN
    energy in the initial state must stop the run after the first step."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(12, 12, bc="periodic")
    st = s.state.copy()
    st[7, 7, 7] = np.nan
    _, _, crashed = oracle.run(s, st, 5)
    assert crashed == 0


def test_oracle_mixed_walls_compose_the_passes(oracle):
    """Periodic x with symmetric y: the x ghosts are periodic copies of the
    interior columns and the y ghosts the symmetric y pass applied after
    them (the order of the reference's boundary calls)."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(12, 10, bc="periodic", bc_y="symmetric")
    u = oracle.boundary(s, s.state)
    nx, ny = s.nx, s.ny
    # x ghosts of interior rows are copies of the wrapped columns
    assert np.array_equal(u[0:3, 3:ny - 3], u[nx - 6:nx - 3, 3:ny - 3])
    assert np.array_equal(u[nx - 3:nx, 3:ny - 3], u[3:6, 3:ny - 3])
    # hydro fields of y ghosts mirror rows 5,4,3
    for f in (0, 1, 2, 3, 6, 7):
        assert np.array_equal(u[:, 0:3, f], u[:, 5:2:-1, f])
    # bY ghosts are not mirrors: integrated from div B = 0 of the first row
    bx, by = u[..., 4], u[..., 5]
    div = (bx[1:, 3] - bx[:-1, 3]) / s.dx + (by[1:, 3] - by[1:, 2]) / s.dy
    assert np.abs(div).max() < 1e-12
