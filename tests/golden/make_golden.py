"""Generate the golden fixtures of tests/golden/ by running the REFERENCE's own
step (keita-akutagawa/ResistiveMHD_GPU single-GPU library, built for the host
by oracle/build_ref.py into oracle/_ref/ref_cpu_{periodic,symmetric}).

Each fixture stores the initial state (boundary not yet applied, as handed to
the reference's initializeU), the solver parameters, the reference's final
state after `steps` RK2 steps and its per-step dt.  Initial states are stored
rather than regenerated so the fixtures do not depend on the host's libm.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import run_reference  # noqa: E402
from resistivemhd_gpu_b200 import setups  # noqa: E402

CASES = {
    # name: (setup factory, steps)
    "ot32_periodic": (lambda: setups.orszag_tang(32), 20),
    "random_periodic_24x18": (lambda: setups.random_smooth_state(24, 18, bc="periodic"), 12),
    "random_symmetric_20x26": (lambda: setups.random_smooth_state(20, 26, bc="symmetric"), 12),
    "random_symmetric_table_22x16": (lambda: setups.random_smooth_state(22, 16, bc="symmetric", with_table=True), 12),
    "harris_64x32": (lambda: setups.harris_sheet(64, 32), 10),
    "ot_minimal_6x6": (lambda: setups.orszag_tang(6), 8),
}


def main() -> None:
    out_dir = Path(__file__).resolve().parent
    for name, (factory, steps) in CASES.items():
        s = factory()
        final, dts, info = run_reference(s, s.state, steps, kind="cpu", threads=1)
        np.savez_compressed(
            out_dir / f"{name}.npz",
            initial=s.state, final=final, dts=dts,
            eta_table=s.eta_table if s.eta_table is not None else np.zeros(0),
            params=np.array([s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta]),
            bc=np.array(s.bc), steps=np.array(steps),
            total_time=np.array(info["total_time"]),
        )
        print(f"{name}: {s.nx}x{s.ny} {steps} steps, total_time {info['total_time']:.6g}")


if __name__ == "__main__":
    main()
