"""The multi-GPU library's walls (ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU/
boundary.cu:48-355) as wall kinds of this library: zero-gradient copies,
the conducting y wall and the flare x wall, in the oracle and in the CUDA
boundary fill, with both CT schemes."""
import dataclasses

import numpy as np
import pytest

# (x walls, y walls): the pairings of the multi-GPU library's step variants
# (resistiveMHD2D.cu:224-454) and mixes with the single-GPU library's walls
PAIRS = [("periodic", "wall"), ("periodic", "zero_gradient"), ("flare", "wall"),
         ("zero_gradient", "zero_gradient"), ("symmetric", "wall"), ("flare", "symmetric")]


def _setup(bcx, bcy, ct="stage1", seed=3, shape=(22, 18), table=False):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=seed, bc=bcx, bc_y=bcy, with_table=table)
    return dataclasses.replace(s, ct=ct)


def test_oracle_wall_semantics(oracle):
    s = _setup("flare", "wall")
    u = oracle.boundary(s, s.state)
    nx, ny, gm = s.nx, s.ny, s.gamma
    # conducting y walls: zero velocity and bY, density, bX, bZ of row 3 / ny-4 (after the x pass)
    for lo, src in ((range(0, 3), 3), (range(ny - 3, ny), ny - 4)):
        for j in lo:
            assert np.all(u[:, j, 1:4] == 0) and np.all(u[:, j, 5] == 0)
            assert np.array_equal(u[:, j, 0], u[:, src, 0])
            assert np.array_equal(u[:, j, 4], u[:, src, 4]) and np.array_equal(u[:, j, 6], u[:, src, 6])
    # flare x = xmin: line-tied (u = w = 0, bY = 0, v kept) from column 3; x = xmax: copies of column nx-4
    r = slice(3, ny - 3)
    for i in range(3):
        assert np.all(u[i, r, 1] == 0) and np.all(u[i, r, 3] == 0) and np.all(u[i, r, 5] == 0)
        assert np.allclose(u[i, r, 2], u[3, r, 2], rtol=1e-15)
        assert np.array_equal(u[nx - 1 - i, r], u[nx - 4, r])
    # the rebuilt energy keeps the source cell's pressure
    c = s.state[3, 5]
    p = (gm - 1) * (c[7] - 0.5 * (c[1] ** 2 + c[2] ** 2 + c[3] ** 2) / c[0] - 0.5 * (c[4] ** 2 + c[5] ** 2 + c[6] ** 2))
    g = u[0, 5]
    assert g[7] == pytest.approx(p / (gm - 1) + 0.5 * g[2] ** 2 / g[0] + 0.5 * (g[4] ** 2 + g[6] ** 2), rel=1e-14)
    z = oracle.boundary(_setup("zero_gradient", "zero_gradient"), s.state)
    assert np.array_equal(z[0:3, 3:ny - 3], np.broadcast_to(z[3:4, 3:ny - 3], (3, ny - 6, 8)))
    assert np.array_equal(z[3:nx - 3, 0:3], np.broadcast_to(z[3:nx - 3, 3:4], (nx - 6, 3, 8)))


@pytest.mark.gpu
@pytest.mark.parametrize("ct", ["stage1", "contact"])
@pytest.mark.parametrize("bcx,bcy", PAIRS)
def test_walls_match_oracle_bit_for_bit(gpu, oracle, bcx, bcy, ct):
    from resistivemhd_gpu_b200 import Solver

    s = _setup(bcx, bcy, ct=ct, table=True)
    n = 6
    ref, rdts, crashed = oracle.run(s, s.state, n)
    assert crashed == -1
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        dts = []
        for _ in range(n):
            sol.step()
            dts.append(sol.dt)
        assert np.array_equal(np.array(dts), rdts)
        assert np.array_equal(sol.get_state(), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("bcx,bcy", PAIRS)
def test_walls_fast_variant_and_batch(gpu, oracle, bcx, bcy):
    from resistivemhd_gpu_b200 import Batch, Solver

    s = _setup(bcx, bcy, shape=(40, 28))
    ref, _, _ = oracle.run(s, s.state, 6)
    with Solver.from_setup(s, precision="fp64_fast") as sol:
        sol.run(6)
        got = sol.get_state()
    for f in range(8):
        den = np.abs(ref[..., f]).sum()
        if den:
            assert np.abs(got[..., f] - ref[..., f]).sum() / den <= 1e-12
    with Batch([s, _setup("periodic", "periodic")], precision="fp64_exact") as b:
        b.run(6)
        assert np.array_equal(b[0].get_state(), ref)


def test_invalid_wall_pairings_are_refused():
    from resistivemhd_gpu_b200 import Solver, _lib

    for bcx, bcy in (("wall", "periodic"), ("periodic", "flare"), ("flare", None)):
        with pytest.raises(_lib.RMHDError) as e:     # checked before any device is touched
            Solver(20, 20, 0.1, 0.1, bc=bcx, bc_y=bcy)
        assert e.value.status == 1                   # RMHD2D_ERR_INVALID
