"""Pins of the parts this library takes from the reference's multi-GPU library
(ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU) against that library's own
code, built unmodified for the host on one rank (oracle/build_ref.py mc):

* its walls (boundary.cu:48-355) in the compositions of its step variants
  (resistiveMHD2D.cu:216-452: sendrecv_U on one rank, then the x and y wall
  functions) against the oracle's ghost fill and the CUDA ghost fill;
* the closing CT of its CT-Contact step (ct.cu:26-257: setOldFlux2D,
  setNowFlux2D, divBClean) against the oracle's restatement
  (orc_contact_ct), which the CUDA CT-Contact step equals bit for bit
  (tests/test_gpu_contact.py).

Golden fixtures (tests/golden/make_golden_mc.py) pin both without the
reference; where oracle/_ref/mc_host is present, fresh random cases are run
against it live.  The rest of the multi-GPU library's step (its fluxes with
the resistive stencil at faces, its dt without the diffusive limit, eta
sampled at (i dx, j dy)) is not this library's arithmetic and stays unpinned.
"""
import dataclasses

import numpy as np
import pytest

from conftest import GOLDEN


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def _setup_from(params, state, bc="periodic", bc_y=None, eta_table=None):
    from resistivemhd_gpu_b200.setups import Setup

    dx, dy, gamma, cfl, eps, eta = (float(v) for v in params)
    return Setup("mc", state.copy(), dx, dy, gamma, cfl, eps, eta, eta_table, bc, bc_y=bc_y)


def _pairs():
    from oracle.oracle import MC_PAIRS

    return sorted(MC_PAIRS)


def _mc_available():
    from oracle.oracle import MC_BINARY

    return MC_BINARY.exists()


# faces whose CT reads corner EMFs built from defined entries only: the
# library leaves the outermost ring of its per-cell EMF inputs unwritten
CT_WINDOW = (slice(2, -3), slice(2, -3))


@pytest.mark.parametrize("pair", _pairs())
def test_oracle_walls_match_mc_golden(oracle, pair):
    from oracle.oracle import MC_PAIRS

    z = np.load(GOLDEN / "mc_walls.npz")
    bx, by = MC_PAIRS[pair]
    s = _setup_from(z["mc_params"], z["state_in"], bx, by)
    assert np.array_equal(_bits(oracle.boundary(s, s.state)), _bits(z[f"{pair}_out"]))


def test_oracle_contact_ct_matches_mc_golden(oracle):
    z = np.load(GOLDEN / "mc_contact_ct.npz")
    s = _setup_from(z["mc_params"], z["u_now"], eta_table=z["eta_table"])
    got = oracle.contact_ct(s, z["u_old"], z["f_old"], z["g_old"], z["u_now"], z["f_now"], z["g_now"], z["bx_old"],
                            z["by_old"], float(z["dt"]))
    assert np.array_equal(_bits(got[CT_WINDOW]), _bits(z["out"][CT_WINDOW]))
    # the CT did change face B, and nothing else
    assert not np.array_equal(got[CT_WINDOW][..., 4:6], z["u_now"][CT_WINDOW][..., 4:6])
    keep = [0, 1, 2, 3, 6, 7]
    assert np.array_equal(_bits(got[..., keep]), _bits(z["u_now"][..., keep]))


@pytest.mark.skipif(not _mc_available(), reason="oracle/_ref/mc_host not built (needs the reference sources)")
@pytest.mark.parametrize("shape,seed", [((9, 7), 1), ((23, 14), 2), ((6, 31), 3)])
def test_oracle_walls_match_mc_live(oracle, shape, seed):
    from oracle.oracle import MC_PAIRS, run_mc_boundary
    from resistivemhd_gpu_b200 import setups

    base = setups.random_smooth_state(*shape, seed=seed, bc="periodic")
    for pair, (bx, by) in MC_PAIRS.items():
        s = dataclasses.replace(base, bc=bx, bc_y=by)
        assert np.array_equal(_bits(oracle.boundary(s, s.state)), _bits(run_mc_boundary(s, s.state, pair))), pair


@pytest.mark.skipif(not _mc_available(), reason="oracle/_ref/mc_host not built (needs the reference sources)")
@pytest.mark.parametrize("shape,seed,table", [((10, 13), 4, False), ((17, 9), 5, True), ((6, 6), 6, True)])
def test_oracle_contact_ct_matches_mc_live(oracle, shape, seed, table):
    from oracle.oracle import run_mc_ct
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*shape, seed=seed, bc="periodic", with_table=table)
    rng = np.random.default_rng(seed)
    sh = s.state.shape
    u_now = s.state * (1.0 + 1e-3 * rng.standard_normal(sh))
    u_now[..., 0] = np.abs(u_now[..., 0])
    f_old, g_old, f_now, g_now = (rng.standard_normal(sh) for _ in range(4))
    # exact zeros in the mass fluxes take the sign() == 0 branch of the upwinding
    f_old[::3, ::2, 0] = 0.0
    g_now[1::4, ::3, 0] = 0.0
    bx_old = s.state[..., 4] + 1e-2 * rng.standard_normal(sh[:2])
    by_old = s.state[..., 5] + 1e-2 * rng.standard_normal(sh[:2])
    args = (s.state, f_old, g_old, u_now, f_now, g_now, bx_old, by_old, 1.7e-3)
    got = oracle.contact_ct(s, *args)
    ref = run_mc_ct(s, *args)
    assert np.array_equal(_bits(got[CT_WINDOW]), _bits(ref[CT_WINDOW]))


@pytest.mark.gpu
@pytest.mark.parametrize("pair", _pairs())
def test_cuda_walls_match_mc_golden(gpu, pair):
    """The CUDA ghost fill (set_state with the boundary applied) on the
    fixture's state equals the multi-GPU library's own fill bit for bit."""
    from oracle.oracle import MC_PAIRS
    from resistivemhd_gpu_b200 import Solver

    z = np.load(GOLDEN / "mc_walls.npz")
    bx, by = MC_PAIRS[pair]
    s = _setup_from(z["mc_params"], z["state_in"], bx, by)
    with Solver.from_setup(s, precision="fp64_exact", apply_boundary=False) as sol:
        sol.set_state(s.state, apply_boundary=True)
        got = sol.get_state()
    assert np.array_equal(_bits(got), _bits(z[f"{pair}_out"]))
