"""Writes plasmoid_degenerate_face.npz: a 20 x 20 cell window of the
8192 x 4096 plasmoid-unstable sheet one step before the FP64-exact run
(the reference's arithmetic) first produces a NaN energy, with that step's
dt.  At the window's centre an x-face's HLLD star denominator
rho (S - u)(S - SM) - bX^2 rounds to exactly 0 (the fast and Alfven waves
meet, |bY| ~ 1e-4), the reference adds only its EPS, and the star
velocities it divides out run into the selected double-star state.

Run on a B200 from the repository root:
    python tests/golden/make_plasmoid_degenerate_face.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

HALF = 10


def main() -> None:
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.plasmoid_sheet(8192, 4096)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.run(900)
        step = 900
        while step < 2000:
            before = sol.get_state()
            dt = sol.calculate_dt()
            sol.step()
            step += 1
            if sol.check_crashed():
                break
        else:
            raise SystemExit("no crash within 2000 steps")
        after = sol.get_state()
    i, j = np.argwhere(~np.isfinite(after[..., 7]))[0]
    win = before[i - HALF:i + HALF, j - HALF:j + HALF].copy()
    bad = np.argwhere(~np.isfinite(after[i - HALF:i + HALF, j - HALF:j + HALF, 7]))
    np.savez_compressed(Path(__file__).with_name("plasmoid_degenerate_face.npz"), window=win, dt=dt, step=step,
                        origin=np.array([i - HALF, j - HALF]), nonfinite=bad,
                        dx=s.dx, dy=s.dy, gamma=s.gamma, eta=s.eta)
    print("crash step", step, "at", (int(i), int(j)), "dt", dt, "non-finite window cells", bad.tolist())


if __name__ == "__main__":
    main()
