"""The reference drivers' main loop with snapshots and the step/time log
(ResistiveMHD_singleGPU_thrust/examples2D/plasmoid/main_plasmoid.cu:297-329),
so notebooks written for the reference's output directories read a run made
here unchanged: directory/name_<step>.bin every record_step steps (the save()
format, byte-identical) and a log of "step,totalTime" lines with the time to
4 significant digits (std::setprecision(4))."""
from __future__ import annotations

import os

from .solver import ResistiveMHD2D, Solver


def _fmt4(x: float) -> str:
    """std::ostream << std::setprecision(4) << x with the default float
    field: %g with 4 significant digits."""
    return "%.4g" % x


def run_like_reference(sim, total_step: int, record_step: int, directoryname: str, filename_without_step: str,
                       log_path: str | None = None, total_time: float = 0.0, echo: bool = True) -> dict:
    """Runs steps 0 .. total_step as the reference's main loop does: every
    record_step steps save and log, then one RK2 step, stopping at the first
    crashed state.  `sim` is a Solver or a ResistiveMHD2D.  Returns
    {"stopped_at": step or total_step + 1, "crashed": bool, "total_time": t}."""
    solver = sim.solver if isinstance(sim, ResistiveMHD2D) else sim
    if not isinstance(solver, Solver):
        raise TypeError("sim must be a Solver or a ResistiveMHD2D")
    os.makedirs(directoryname, exist_ok=True)
    log_path = log_path or os.path.join(directoryname, f"log_{filename_without_step}.txt")
    crashed = False
    step = total_step + 1
    with open(log_path, "a") as log:
        for s in range(total_step + 1):
            if s % record_step == 0:
                solver.save(directoryname, filename_without_step, s)
                log.write(f"{s},{_fmt4(total_time)}\n")
                log.flush()
                if echo:
                    print(f"{s} step done : total time is {_fmt4(total_time)}", flush=True)
            solver.step()
            if solver.check_crashed():
                if echo:
                    print(f"Calculation stopped! : {s} steps", flush=True)
                crashed = True
                step = s
                break
            total_time += solver.dt
    return {"stopped_at": step, "crashed": crashed, "total_time": total_time}
