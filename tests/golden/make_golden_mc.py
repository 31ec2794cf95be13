"""Generate the multi-GPU-library fixtures of tests/golden/ by running the
REFERENCE's own code: the wall functions and the CT-Contact closing CT of
keita-akutagawa/ResistiveMHD_GPU's ResistiveMHD_multiGPU_cuda/ResistiveMHD2D_GPU
(boundary.cu, ct.cu, mpi.cu), built unmodified for the host on one rank by
oracle/build_ref.py (`python oracle/build_ref.py mc` -> oracle/_ref/mc_host).

* mc_walls.npz: for each wall pair of the library's step variants, a state
  before and after the library's ghost fill (sendrecv_U on one rank, then its
  x and y wall functions).
* mc_contact_ct.npz: the inputs of CT::setOldFlux2D / setNowFlux2D /
  divBClean (two stages' states and flux records, the step input's face B,
  dt, a cell-centred eta table) and the state the library writes.

Inputs are stored, so the fixtures do not depend on the generator's random
streams or the host's libm.

    python tests/golden/make_golden_mc.py
"""
from __future__ import annotations

import dataclasses
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import MC_PAIRS, run_mc_boundary, run_mc_ct  # noqa: E402
from resistivemhd_gpu_b200 import setups  # noqa: E402

OUT = Path(__file__).resolve().parent


def contact_inputs(nx_int: int, ny_int: int, seed: int):
    """A smooth state with an eta table and two stages' inputs: the second
    stage's state a perturbation of the first, flux records of both signs."""
    s = setups.random_smooth_state(nx_int, ny_int, seed=seed, bc="periodic", with_table=True)
    rng = np.random.default_rng(seed)
    sh = s.state.shape
    u_old = s.state.copy()
    u_now = s.state * (1.0 + 1e-3 * rng.standard_normal(sh))
    u_now[..., 0] = np.abs(u_now[..., 0])
    f_old, g_old, f_now, g_now = (rng.standard_normal(sh) for _ in range(4))
    bx_old = s.state[..., 4] + 1e-2 * rng.standard_normal(sh[:2])
    by_old = s.state[..., 5] + 1e-2 * rng.standard_normal(sh[:2])
    return s, dict(u_old=u_old, f_old=f_old, g_old=g_old, u_now=u_now, f_now=f_now, g_now=g_now, bx_old=bx_old,
                   by_old=by_old)


def main() -> None:
    w = setups.random_smooth_state(14, 12, seed=21, bc="periodic")
    walls = {"state_in": w.state}
    for pair, (bx, by) in MC_PAIRS.items():
        walls[f"{pair}_out"] = run_mc_boundary(dataclasses.replace(w, bc=bx, bc_y=by), w.state, pair)
    np.savez_compressed(OUT / "mc_walls.npz", mc_params=np.array([w.dx, w.dy, w.gamma, w.cfl, w.eps, w.eta]),
                        **walls)
    s, inp = contact_inputs(12, 10, seed=22)
    dt = 2.5e-3
    out = run_mc_ct(s, dt=dt, **inp)
    np.savez_compressed(OUT / "mc_contact_ct.npz", mc_params=np.array([s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta]),
                        dt=np.array(dt), eta_table=s.eta_table, out=out, **inp)
    print(f"mc_walls.npz: {len(MC_PAIRS)} pairs on {w.nx}x{w.ny}; mc_contact_ct.npz on {s.nx}x{s.ny}")


if __name__ == "__main__":
    main()
