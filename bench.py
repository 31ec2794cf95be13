#!/usr/bin/env python
"""Benchmark of the B200 resistive-MHD RK2 step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64_exact|fp64_fast|fp32_bulk] [--workload harris|orszag_tang]

Workload (default): the Harris current sheet, 2048 x 1024 interior cells,
symmetric walls, uniform eta 1e-3 plus a Gaussian eta bump (cell-centred
table), FP64 -- the configuration the headline metric is quoted on.  The
headline precision is fp64_exact, the drop-in: bit-identical to the
reference's IEEE binary64 arithmetic.  fp64_fast (FMA contraction, shared
reciprocals) and fp32_bulk are reported beside it with their relative L1
against fp64_exact at the same dts.  A
"step" is one full RK2 step (two fused stage kernels, two boundary fills,
the CFL reduction for the next dt).  The state (2 x 135 MB) is larger than
the 126 MB L2, so no L2 flush is needed between steps.

Metric: interior cell-updates per second (higher is better).

--impl reference times the reference's own step (the unmodified library of
keita-akutagawa/ResistiveMHD_GPU built for the host with Thrust's OpenMP
backend by oracle/build_ref.py) on all host cores, on the same workload.

For --gpus N > 1 (launched with torch.distributed.run) each rank runs an
independent replica of the workload on its own GPU ("replicas only": the
single-domain step has no exchange), value = all ranks' cell-updates / the
slowest rank's device time.

Extra blocks of the same JSON line (each can be switched off):
  precision  FP32-bulk vs FP64 (fast and exact) on the headline workload:
             throughput of each, and the relative L1 error of rho, p, B and
             J_z against the FP64-exact run at the same dts.
  adjoint    the discrete adjoint on the adjoint workload (512^2 periodic
             Orszag-Tang, eta = 1e-3 exp(g/2) with g a Gaussian random field
             of correlation length 0.3, 2000 steps, sqrt(N) checkpoints):
             forward, recorded forward and backward times and their ratios
             for the FP32-bulk and FP64 forwards, and central differences
             (h = 1e-6) through the FP64 forward on 32 seeded directions.
  ct_contact the CT-Contact step (cfg.ct_scheme) on the headline workload
             against the stage-1-EMF step, both in FP64 without contraction.
  ensemble   256 independent periodic runs (Orszag-Tang / Kelvin-Helmholtz,
             n^2 with n in {128..512}, eta log-uniform in [1e-4, 1e-2], 500
             steps) in one persistent batch in FP32-bulk, against the FP64
             path looped one run at a time; with N > 1 the runs are sharded
             over the ranks (no collective on the data path).
  ref_gpu    the reference's own library built for sm_100a on the same GPU,
             timed with CUDA events inside its driver, and the relative L1
             of its final state against fp64_exact after the same steps;
             ref_gpu_2048sq the same on a 2048 x 2048 periodic Orszag-Tang
             grid.
  summary    the figures above in a few keys, last in the line.

--study harris|plasmoid replaces the benchmark with the long error study of
FP32-bulk against FP64 at the same dts, beside an FP64 run that differs from
the reference by round-off only: Harris 2048 x 1024 for 5000 steps against
the drop-in, or the plasmoid-unstable sheet 8192 x 4096 (half-width 0.1, eta
1e-5, beta 0.1) for 20000 steps against fp64_fast, with the relative L1 of
rho, p, B and J_z and max |div B| at 5 evenly spaced snapshots.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "cell-updates/s"
MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def workload(name: str):
    from resistivemhd_gpu_b200 import setups

    if name == "harris":
        return setups.harris_sheet(2048, 1024), "harris_2048x1024"
    if name == "orszag_tang":
        return setups.orszag_tang(256), "orszag_tang_256x256"
    raise SystemExit(f"unknown workload {name}")


def algorithmic_bytes(setup) -> dict:
    """Minimum HBM bytes per launch of each stage kernel.
    stage 1 reads U^n (8 doubles/cell) [+ eta], writes U* (8);
    stage 2 reads U* (8) and the hydro part of U^n (6) [+ eta], writes U^{n+1} (8)."""
    cells = setup.interior_cells
    eta = 8 if setup.eta_table is not None else 0
    return {"stage1": cells * (64 + 64 + eta), "stage2": cells * (64 + 48 + 64 + eta), "per_cell_update":
            (64 + 64 + eta) + (64 + 48 + 64 + eta)}


def hbm_peak():
    try:
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


B200_FP64_TFLOPS_NOMINAL_PIPE = 148 * 64 * 2 * 1.965e9 / 1e12   # SMs x FP64 FMA lanes x 2 x max clock
# sizeof(rmhd2d::Control): the control block each synchronising query (crash flag, dt) reads back
CONTROL_BLOCK_BYTES = 64


def flops_from_profile(label: str):
    """Floating-point operations per cell-update of the algorithm, from the
    committed count (profiles/flops_<label>.md, line
    'flops_per_cell_update:')."""
    p = ROOT / "profiles" / f"flops_{label}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("flops_per_cell_update:"):
            return float(line.split(":", 1)[1])
    return None


def traffic_from_profile(label: str):
    """dram bytes per launch of the stage kernels from the committed ncu
    summary (profiles/stage_kernel_<label>.md, line 'traffic_bytes_per_launch:')."""
    p = ROOT / "profiles" / f"stage_kernel_{label}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            vals = dict(kv.split("=") for kv in line.split(":", 1)[1].split())
            return {k: float(v) for k, v in vals.items()}
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.tmp = tempfile.NamedTemporaryFile(prefix="clk", suffix=".csv", delete=False)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.tmp, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        try:
            rows = [r.split(",") for r in Path(self.tmp.name).read_text().strip().splitlines() if r.strip()]
            os.unlink(self.tmp.name)
        except Exception:
            rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], None, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except Exception:
                continue
        loaded = [v for v in sm if mx and v > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_reference_binary(kind: str, setup, warmup: int, steps: int, threads: int | None):
    from oracle.oracle import run_reference

    _, _, info = run_reference(setup, setup.state, steps, n_warmup=warmup, kind=kind, threads=threads,
                               timeout=3600)
    return info


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def workload_config(setup, label: str, precision: str, world: int) -> dict:
    """The config object of the JSON line, the same for both arms."""
    return {"workload": label, "cells": setup.interior_cells, "nx": setup.nx, "ny": setup.ny, "bc": setup.bc,
            "eta": "uniform 1e-3 + gaussian bump (cell-centred table)" if setup.eta_table is not None
            else f"uniform {setup.eta}",
            "precision": precision, "parallelism": f"replicas x{world}" if world > 1 else "single",
            "l2": "inputs larger than L2 (2 x state = %.0f MB)" % (2 * setup.state.nbytes / 1e6)}


def reference_arm(args, rank: int) -> None:
    if rank != 0:
        return
    setup, label = workload(args.workload)
    threads = os.cpu_count() or 1
    info = run_reference_binary("cpu", setup, args.warmup, args.steps, threads)
    secs = info["seconds"]
    value = setup.interior_cells * args.steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(setup, label, args.precision, 1),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "reference",
                         "sample": f"{label}: {args.warmup} warm-up + {args.steps} timed steps of the reference "
                                   f"library built for the host (Thrust OMP backend) on {threads} threads, "
                                   f"{cpu_model()}"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ours_arm(args, rank: int, world: int, local_rank: int) -> None:
    import numpy as np
    import torch

    from resistivemhd_gpu_b200 import Solver

    torch.cuda.set_device(local_rank)
    setup, label = workload(args.workload)
    dist = None
    if world > 1:
        import torch.distributed as dist  # noqa: F811

    sol = Solver.from_setup(setup, precision=args.precision, device=local_rank)
    # the stage kernels' tile shape, picked by the library's autotuner on this
    # workload (the state is restored afterwards; results do not depend on
    # it), unless given (a profiler run that must launch what the timed run did)
    if args.tile_shapes:
        sol.set_stage_shapes(*args.tile_shapes)
        tuning = {}
    else:
        sol.autotune(6)
        tuning = sol.tuning()
    shape = list(sol.stage_shapes)
    sol.run(args.warmup)
    sol.dt  # synchronise

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-timed region: exactly K steps ----
    barrier()
    with ClockSampler(local_rank) as clk:
        ms = sol.run_timed(args.steps)
    barrier()
    crashed = sol.check_crashed()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    cells = setup.interior_cells
    value = world * cells * args.steps / (ms_max * 1e-3)

    # ---- per-kernel breakdown for the roofline (same stream, CUDA events) ----
    prof = [sol.profile_step() for _ in range(max(3, min(args.steps, 20)))]
    st1 = statistics.median(p[0] for p in prof)
    bn1 = statistics.median(p[1] for p in prof)
    st2 = statistics.median(p[2] for p in prof)
    bn2 = statistics.median(p[3] for p in prof)
    ab = algorithmic_bytes(setup)
    peak, peak_kind = hbm_peak()
    achieved = (ab["stage1"] + ab["stage2"]) / ((st1 + st2) * 1e-3) / 1e9
    traffic = traffic_from_profile(f"{label}_{args.precision}")
    roofline = {
        "kernel": "stage_kernel (stage 1 + stage 2 per step)", "bound": "hbm", "achieved": achieved,
        "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
        "traffic": (traffic["stage1"] + traffic["stage2"]) / 2 if traffic else None,
        "algorithmic_bytes_per_launch": (ab["stage1"] + ab["stage2"]) / 2,
        "launch_ms": {"stage1": st1, "boundary1": bn1, "stage2": st2, "boundary2_cfl": bn2},
        "note": "FP64-issue bound: the fp64 object carries the FP64 roofline",
    }

    # ---- end-to-end through the public API with pinned host buffers ----
    e2e = None
    if args.e2e:
        host = torch.empty(setup.state.shape, dtype=torch.float64, pin_memory=True).numpy()
        host[...] = setup.state
        out = torch.empty(setup.state.shape, dtype=torch.float64, pin_memory=True).numpy()
        e2e_sol = Solver(setup.nx, setup.ny, setup.dx, setup.dy, gamma=setup.gamma, cfl=setup.cfl, eps=setup.eps,
                         eta=setup.eta, bc=setup.bc, precision=args.precision, device=local_rank)
        if setup.eta_table is not None:
            e2e_sol.set_eta_table(setup.eta_table)
        e2e_sol.set_state(host, apply_boundary=True)
        e2e_sol.run(args.warmup)
        e2e_sol.dt
        barrier()
        t0 = time.perf_counter()
        e2e_sol.set_state(host, apply_boundary=True)          # H2D of the initial state
        total = 0.0
        for _ in range(args.steps):
            e2e_sol.step()                                     # oneStepRK2
            if e2e_sol.check_crashed():                        # checkCalculationIsCrashed (D2H)
                break
            total += e2e_sol.dt                                # totalTime += dt (D2H)
        e2e_sol.get_state(out)                                 # getU (D2H of the result)
        t1 = time.perf_counter()
        el = torch.tensor([t1 - t0], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(el, op=dist.ReduceOp.MAX)
        state_bytes = setup.state.nbytes
        e2e = {"value": world * cells * args.steps / float(el.item()), "unit": METRIC,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": state_bytes / args.steps + 2 * CONTROL_BLOCK_BYTES,
               "note": "set_state(pinned) + K x (step_rk2 + check_crashed + get_dt) + get_state(pinned), wall clock"}
        e2e_sol.close()

    line = None
    if rank == 0:
        clocks = clk.summary()
        gpu_launches = 4 * args.steps
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if args.precision == "fp32_bulk" else "f64", "data": "synthetic",
            "config": workload_config(setup, label, args.precision, world),
            "roofline": roofline,
            "clocks": clocks,
            "tile_shapes": shape,
            "headline_tuning": {f"shape_{k}": {"stage1_ms": v[0], "stage2_ms": v[1]} for k, v in tuning.items()},
            "gpu_launches": gpu_launches,
            "crashed": crashed,
        }
        if e2e:
            line["e2e"] = e2e
        # The FP64 roofline beside the HBM one: the algorithm's flops per
        # cell-update (counted on the oracle's operation-counting scalar,
        # profiles/flops_<label>.md) times the measured rate, against the
        # nominal FP64 pipe rate (the measured peaks file has no FP64 figure).
        fpc = flops_from_profile(label)
        achieved_tf = None if fpc is None else fpc * value / world / 1e12   # per GPU
        line["fp64"] = {"bound": "fp64", "flops_per_cell_update": fpc, "achieved_tflops": achieved_tf,
                        "peak_tflops": B200_FP64_TFLOPS_NOMINAL_PIPE,
                        "peak_kind": "nominal: 148 SMs x 64 FP64 FMA lanes x 2 x 1.965 GHz",
                        "frac": None if achieved_tf is None else achieved_tf / B200_FP64_TFLOPS_NOMINAL_PIPE,
                        "flops_source": f"profiles/flops_{label}.md",
                        "pipe_counters": f"profiles/stage_kernel_{label}_{args.precision}.md"}
    sol.close()

    if rank == 0 and world == 1 and args.baselines:
        # reference's own CUDA build on the same GPU (bounded sample), timed
        # with CUDA events around its step loop inside the reference driver
        try:
            line["ref_gpu"] = ref_gpu_block(setup, label, value, local_rank)
        except Exception as e:  # reported, never fatal
            line["ref_gpu"] = {"unavailable": str(e)[:200]}
        # the same comparison on a square 2048^2 grid (periodic Orszag-Tang)
        try:
            line["ref_gpu_2048sq"] = ref_gpu_square_block(local_rank)
        except Exception as e:  # reported, never fatal
            line["ref_gpu_2048sq"] = {"unavailable": str(e)[:200]}
        # reference's own CPU build on the host cores (bounded sample)
        try:
            threads = os.cpu_count() or 1
            k = 6
            info = run_reference_binary("cpu", setup, 1, k, threads)
            cv = cells * k / info["seconds"]
            line["cpu_baseline"] = {"value": cv, "unit": METRIC, "cores": threads, "kind": "reference",
                                    "sample": f"{label}: 1 warm-up + {k} timed steps of the reference library built "
                                              f"for the host (Thrust OMP backend), {threads} threads, {cpu_model()}"}
        except Exception as e:
            line["cpu_baseline"] = {"unavailable": str(e)[:200]}
    if world == 1 and args.precision_block:
        line["precision"] = precision_block(args, setup, label, local_rank)
    if world == 1 and args.contact_block:
        line["ct_contact"] = contact_block(args, setup, label, local_rank)
    if world == 1 and args.adjoint_block:
        line["adjoint"] = adjoint_block(args, local_rank)
    if args.ensemble_block:
        ens = ensemble_block(args, rank, world, local_rank, dist)
        if line is not None:
            line["ensemble"] = ens
    if line is not None:
        line["summary"] = summary_of(line)
        print(json.dumps(line), flush=True)


def summary_of(line: dict) -> dict:
    """The figures of the extra blocks in a few keys, placed last in the
    line so that they sit in the end of the output that a log tail keeps."""
    out = {"headline_precision": line["config"]["precision"], "value": line["value"],
           "ms_per_step": line["ms_per_step"], "roofline_frac": line["roofline"]["frac"]}
    pr = line.get("precision")
    if pr:
        for prec in ("fp64_exact", "fp64_fast", "fp32_bulk"):
            out[f"{prec}_value"] = pr[prec]["value"]
            out[f"{prec}_ms_per_step"] = pr[prec]["ms_per_step"]
            if "rel_l1" in pr[prec]:
                out[f"{prec}_max_rel_l1_vs_exact"] = max(pr[prec]["rel_l1"][k] for k in ("rho", "p", "B"))
        out["error_steps"] = pr.get("error_steps")
        out["fp32_bulk_over_fp64_fast"] = pr["bulk_speedup_vs_fp64_fast"]
        out["fp32_bulk_over_fp64_exact"] = pr["bulk_speedup_vs_fp64_exact"]
    rg = line.get("ref_gpu")
    if rg and "value" in rg:
        out["ref_gpu_value"] = rg["value"]
        out["speedup_vs_ref_gpu"] = rg["speedup"]
        out["ref_gpu_vs_ref_host_max_rel_l1"] = rg.get("vs_fp64_exact_max_rel_l1")
    rq = line.get("ref_gpu_2048sq")
    if rq and "value" in rq:
        out["speedup_vs_ref_gpu_2048sq"] = rq["speedup"]
    cb = line.get("cpu_baseline")
    if cb and "value" in cb:
        out["cpu_baseline_value"] = cb["value"]
    ad = line.get("adjoint")
    if ad:
        for prec in ("fp32_bulk", "fp64_exact", "fp32_bulk_whole_trajectory", "fp64_exact_whole_trajectory"):
            if prec in ad and "adjoint_over_forward" in ad[prec]:
                out[f"adjoint_over_forward_{prec}"] = ad[prec]["adjoint_over_forward"]
        for key in ("fd", "fd_smooth_control"):
            if key in ad and "frac_le_1e-6" in ad[key]:
                out[f"adjoint_{key}_frac_le_1e-6"] = ad[key]["frac_le_1e-6"]
        for hk, hv in ad.get("fd_noisy_start", {}).items():
            if isinstance(hv, dict) and "frac_le_1e-6" in hv:
                out[f"adjoint_fd_{hk}_frac_le_1e-6"] = hv["frac_le_1e-6"]
                out[f"adjoint_fd_{hk}_rel_err_median"] = hv["rel_err_median"]
                out[f"adjoint_fd_{hk}_taylor_slope"] = hv["taylor_remainder_slope_median"]
        for hk, hv in ad.get("bulk_forward_gradient_vs_horizon", {}).items():
            out[f"adjoint_bulk_gradient_rel_l2_{hk}"] = hv["state"]
    en = line.get("ensemble")
    if en and "speedup_vs_loop_fp64" in en:
        out["ensemble_value"] = en["batch_fp32_bulk"]["value"]
        out["ensemble_speedup_vs_loop_fp64"] = en["speedup_vs_loop_fp64"]
    if en and "autotune" in en:
        out["ensemble_autotune_chosen"] = en["autotune"]["chosen"]
        out["ensemble_autotune_margin_over_default"] = en["autotune"]["margin_over_default"]
    if "tile_shapes" in line:
        out["headline_tile_shapes"] = line["tile_shapes"]
    ct = line.get("ct_contact")
    if ct:
        out["ct_contact_over_stage1_time"] = ct["contact_over_stage1_time"]
    return out


def ref_gpu_block(setup, label, value, local_rank, warmup=2, steps=20):
    """The reference's own library built for sm_100a (nvcc -O3, contraction
    on, as its example makefiles build it) on the same GPU: throughput from
    CUDA events around its oneStepRK2 + checkCalculationIsCrashed loop, and
    how far its final state lies from this library's FP64-exact step (the
    reference's IEEE arithmetic without contraction) after the same steps."""
    import numpy as np

    from resistivemhd_gpu_b200 import Solver

    ref_state, ref_dts, info = _reference_run("gpu", setup, warmup, steps)
    secs = info["event_seconds"] if info.get("event_seconds", -1) > 0 else info["seconds"]
    rv = setup.interior_cells * info["steps"] / secs
    with Solver.from_setup(setup, precision="fp64_exact", device=local_rank) as sol:
        for _ in range(len(ref_dts)):
            sol.step()
        ours = sol.get_state()
    d_ref = _diagnostics(ref_state, setup.dx, setup.dy, setup.gamma)
    d_our = _diagnostics(ours, setup.dx, setup.dy, setup.gamma)
    err = {k: _rel_l1(d_ref[k], d_our[k]) for k in d_ref}
    return {"value": rv, "unit": METRIC, "speedup": value / rv, "ms_per_step": 1e3 * secs / info["steps"],
            "timing": "CUDA events on the legacy default stream around the timed steps",
            "wall_ms_per_step": 1e3 * info["seconds"] / info["steps"],
            "vs_fp64_exact_rel_l1": err, "vs_fp64_exact_max_rel_l1": max(err[k] for k in ("rho", "p", "B")),
            "vs_fp64_exact_steps": len(ref_dts),
            "sample": f"{label}: {warmup} warm-up + {info['steps']} steps of the reference library built for "
                      "sm_100a (nvcc -O3, FMA contraction on; oneStepRK2 + checkCalculationIsCrashed)"}


def ref_gpu_square_block(local_rank, n=2048, warmup=2, steps=10):
    """This library's fp64_exact step against the reference's sm_100a build
    on the same GPU, on a 2048 x 2048 periodic Orszag-Tang grid."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.orszag_tang(n)
    with Solver.from_setup(s, precision="fp64_exact", device=local_rank) as sol:
        sol.autotune(4)
        sol.run(warmup)
        ms = sol.run_timed(steps)
    ours = s.interior_cells * steps / (ms * 1e-3)
    blk = ref_gpu_block(s, f"orszag_tang_{n}x{n}", ours, local_rank, warmup=warmup, steps=steps)
    blk["ours_fp64_exact_value"] = ours
    blk["ours_ms_per_step"] = ms / steps
    return blk


def _reference_run(kind, setup, warmup, steps, threads=None):
    from oracle.oracle import run_reference

    return run_reference(setup, setup.state, steps, n_warmup=warmup, kind=kind, threads=threads, timeout=3600)


def _diagnostics(state, dx, dy, gamma):
    """rho, p, bX, bY, bZ and the corner J_z of the interior of a state."""
    u = state[3:-3, 3:-3]
    rho = u[..., 0]
    bxc = 0.5 * (state[3:-3, 3:-3, 4] + state[2:-4, 3:-3, 4])
    byc = 0.5 * (state[3:-3, 3:-3, 5] + state[3:-3, 2:-4, 5])
    ke = 0.5 * (u[..., 1] ** 2 + u[..., 2] ** 2 + u[..., 3] ** 2) / rho
    p = (gamma - 1.0) * (u[..., 7] - ke - 0.5 * (bxc ** 2 + byc ** 2 + u[..., 6] ** 2))
    jz = (state[4:-2, 3:-3, 5] - state[3:-3, 3:-3, 5]) / dx - (state[3:-3, 4:-2, 4] - state[3:-3, 3:-3, 4]) / dy
    return {"rho": rho, "p": p, "B": u[..., 4:7], "J_z": jz}


def _rel_l1(a, b) -> float:
    import numpy as np

    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def precision_block(args, setup, label, local_rank):
    """FP32-bulk against FP64 on the headline workload."""
    from resistivemhd_gpu_b200 import Solver

    nerr = max(args.steps, 100)
    out = {"workload": label, "steps": args.steps, "error_steps": nerr,
           "error_reference": f"fp64_exact at the same dts after {nerr} steps"}
    with Solver.from_setup(setup, precision="fp64_exact", device=local_rank) as ref:
        dts = []
        for _ in range(nerr):
            ref.step()
            dts.append(ref.dt)
        ref_diag = _diagnostics(ref.get_state(), setup.dx, setup.dy, setup.gamma)
    for prec in ("fp64_exact", "fp64_fast", "fp32_bulk"):
        with Solver.from_setup(setup, precision=prec, device=local_rank) as sol:
            sol.autotune(4)
            sol.run(args.warmup)
            ms = sol.run_timed(args.steps)
            entry = {"value": setup.interior_cells * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
                     "tile_shapes": list(sol.stage_shapes)}
            if prec != "fp64_exact":
                sol.set_state(setup.state, apply_boundary=True)
                sol.run_fixed_dt(dts)
                d = _diagnostics(sol.get_state(), setup.dx, setup.dy, setup.gamma)
                entry["rel_l1"] = {k: _rel_l1(d[k], ref_diag[k]) for k in d}
                entry["rel_l1_B_components"] = {c: _rel_l1(d["B"][..., q], ref_diag["B"][..., q])
                                                for q, c in enumerate(("bX", "bY", "bZ"))}
            out[prec] = entry
    out["bulk_speedup_vs_fp64_fast"] = out["fp32_bulk"]["value"] / out["fp64_fast"]["value"]
    out["bulk_speedup_vs_fp64_exact"] = out["fp32_bulk"]["value"] / out["fp64_exact"]["value"]
    out["bulk_max_rel_l1"] = max(out["fp32_bulk"]["rel_l1"].values())
    return out


STUDIES = {
    # name: (setup factory, label, steps, snapshots, FP64 reference precision)
    "harris": (lambda s: s.harris_sheet(2048, 1024), "harris_2048x1024", 5000, 5, "fp64_exact"),
    "plasmoid": (lambda s: s.plasmoid_sheet(8192, 4096), "plasmoid_8192x4096", 20000, 5, "fp64_fast"),
}


def _max_div_b(state, dx, dy) -> float:
    """max |div B| over the interior cells, from the face fields."""
    import numpy as np

    div = (state[3:-3, 3:-3, 4] - state[2:-4, 3:-3, 4]) / dx + (state[3:-3, 3:-3, 5] - state[3:-3, 2:-4, 5]) / dy
    return float(np.abs(div).max())


def precision_study(args, local_rank):
    """FP32-bulk against an FP64 reference run over the full length of a
    workload, at evenly spaced snapshots, beside a "floor" run that differs
    from the reference by round-off only: on Harris the reference is the
    drop-in (fp64_exact) and the floor fp64_fast; on the plasmoid sheet the
    drop-in stops at a degenerate HLLD face (see `drop_in`), so the reference
    is fp64_fast and the floor fp64_fast from a start whose momenta are
    scaled by 1 + 1e-15.  The runs advance in lockstep: the reference takes
    its CFL dts segment by segment and the others replay them
    (rmhd2d_run_fixed_dt), so every snapshot compares the same times.  The
    floor run's error is what the flow's instability makes of round-off;
    FP32-bulk's error is read against it."""
    import numpy as np

    from resistivemhd_gpu_b200 import Solver, setups

    make, label, nsteps, nsnap, ref_prec = STUDIES[args.study]
    if args.study_steps:
        nsteps = args.study_steps
    setup = make(setups)
    seg = [nsteps * (q + 1) // nsnap - nsteps * q // nsnap for q in range(nsnap)]
    floor_prec = "fp64_fast"
    floor_start = setup.state
    floor_desc = "fp64_fast"
    if ref_prec != "fp64_exact":
        floor_start = setup.state.copy()
        floor_start[3:-3, 3:-3, 1:3] *= 1.0 + 1e-15
        floor_desc = "fp64_fast from momenta scaled by 1 + 1e-15"
    out = {"study": label, "steps": nsteps, "snapshots": [], "reference": f"{ref_prec} (its own CFL dts)",
           "floor": floor_desc, "unit": "relative L1 over the interior at the same dts", "data": "synthetic"}
    if ref_prec != "fp64_exact":
        # how far the drop-in (the reference's arithmetic) gets on its own dts
        with Solver.from_setup(setup, precision="fp64_exact", device=local_rank) as ex:
            crashed_at = None
            for q in range(nsteps):
                ex.step()
                if (q + 1) % 50 == 0 and ex.check_crashed():
                    crashed_at = q + 1
                    break
            out["drop_in"] = {"precision": "fp64_exact", "first_crash_check_failed_at_step": crashed_at,
                              "checked_every": 50}
    sols = {"reference": Solver.from_setup(setup, precision=ref_prec, device=local_rank),
            "floor": Solver.from_setup(setup, precision=floor_prec, device=local_rank, apply_boundary=False),
            "fp32_bulk": Solver.from_setup(setup, precision="fp32_bulk", device=local_rank)}
    sols["floor"].set_state(floor_start, apply_boundary=True)
    try:
        done, t_wall = 0, {p: 0.0 for p in sols}
        for n in seg:
            dts = np.empty(n)
            t0 = time.perf_counter()
            for q in range(n):
                sols["reference"].step()
                dts[q] = sols["reference"].dt
            t_wall["reference"] += time.perf_counter() - t0
            for p in ("floor", "fp32_bulk"):
                t0 = time.perf_counter()
                sols[p].run_fixed_dt(dts)
                sols[p].check_crashed()   # synchronises
                t_wall[p] += time.perf_counter() - t0
            done += n
            ref_state = sols["reference"].get_state()
            ref = _diagnostics(ref_state, setup.dx, setup.dy, setup.gamma)
            snap = {"step": done, "time": sols["reference"].total_time,
                    "max_div_b": {"reference": _max_div_b(ref_state, setup.dx, setup.dy)},
                    "crashed": {"reference": sols["reference"].check_crashed()}}
            del ref_state
            for p in ("floor", "fp32_bulk"):
                st = sols[p].get_state()
                d = _diagnostics(st, setup.dx, setup.dy, setup.gamma)
                snap[p] = {k: _rel_l1(d[k], ref[k]) for k in d}
                snap["max_div_b"][p] = _max_div_b(st, setup.dx, setup.dy)
                snap["crashed"][p] = sols[p].check_crashed()
                del st, d
            out["snapshots"].append(snap)
            print(json.dumps({"progress": snap}), file=sys.stderr, flush=True)
        out["wall_s"] = t_wall
    finally:
        for s in sols.values():
            s.close()
    last = out["snapshots"][-1]
    out["final_bulk_over_floor"] = {k: last["fp32_bulk"][k] / max(last["floor"][k], 1e-300)
                                    for k in last["fp32_bulk"]}
    return out


def _misfit_difference(final_p, final_m, target, fields) -> float:
    """J(final_p) - J(final_m) for J = 0.5 sum over the interior of
    (final - target)^2 on `fields`, formed as sum (f_p - f_m) (mean - target):
    the same number as the difference of the two sums, without subtracting
    two large misfits (a localized direction moves J by a tiny fraction of
    it, and J's own rounding would swamp the central difference)."""
    fp = final_p[3:-3, 3:-3, fields]
    fm = final_m[3:-3, 3:-3, fields]
    t = target[3:-3, 3:-3, fields]
    return float(((fp - fm) * (0.5 * (fp + fm) - t)).sum())


def adjoint_block(args, local_rank, n=512, nsteps=2000, ndirs=32, h=1e-6):
    """Cost and finite-difference agreement of the discrete adjoint."""
    import numpy as np

    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.ot_adjoint(n)
    label = f"ot_adjoint_{n}x{n}_{nsteps}steps"
    fields = [0, 4, 5, 6]
    # observation: the same start evolved with uniform eta = 1e-3
    with Solver.from_setup(setups.orszag_tang(n), precision="fp64_exact", device=local_rank) as obs:
        obs.run(nsteps)
        target = obs.get_state()

    def misfit_and_seed(final):
        d = np.zeros_like(final)
        d[3:-3, 3:-3, fields] = final[3:-3, 3:-3, fields] - target[3:-3, 3:-3, fields]
        return 0.5 * float((d * d).sum()), d

    out = {"workload": label, "checkpoint_interval": int(np.ceil(np.sqrt(nsteps))),
           "misfit": "0.5 sum over the interior of ((rho, bX, bY, bZ)(T) - observation)^2",
           "dt": "recorded by the forward run and held fixed"}
    grads = {}
    for prec in ("fp32_bulk", "fp64_exact"):
        with Solver.from_setup(s, precision=prec, device=local_rank) as sol:
            sol.autotune(4)
            sol.run(3)
            sol.set_state(s.state, apply_boundary=True)
            ms_fwd = sol.run_timed(nsteps)
            sol.set_state(s.state, apply_boundary=True)
            sol.adjoint_forward(nsteps)                        # allocates the workspace
            sol.set_state(s.state, apply_boundary=True)
            t0 = time.perf_counter()
            sol.adjoint_forward(nsteps)
            t_rec = time.perf_counter() - t0
            J, seed = misfit_and_seed(sol.get_state())
            t0 = time.perf_counter()
            gs, ge = sol.adjoint_backward(seed)
            t_bwd = time.perf_counter() - t0
            grads[prec] = (gs, ge, sol.adjoint_dts(), J)
            out[prec] = {"forward_ms": ms_fwd, "recorded_forward_ms": 1e3 * t_rec, "backward_ms": 1e3 * t_bwd,
                         "backward_over_forward": 1e3 * t_bwd / ms_fwd,
                         "adjoint_over_forward": 1e3 * (t_rec + t_bwd) / ms_fwd, "misfit": J}
    # the same runs with the whole trajectory kept in HBM (every step's U^n
    # and U*, 2 x 2000 states): the backward recomputes nothing
    for prec in ("fp32_bulk", "fp64_exact"):
        try:
            with Solver.from_setup(s, precision=prec, device=local_rank) as sol:
                sol.autotune(4)
                sol.adjoint_forward(nsteps, -1)                        # allocates the trajectory
                sol.set_state(s.state, apply_boundary=True)
                t0 = time.perf_counter()
                sol.adjoint_forward(nsteps, -1)
                t_rec = time.perf_counter() - t0
                J, seed = misfit_and_seed(sol.get_state())
                t0 = time.perf_counter()
                gs, ge = sol.adjoint_backward(seed)
                t_bwd = time.perf_counter() - t0
                ms_fwd = out[prec]["forward_ms"]
                out[f"{prec}_whole_trajectory"] = {
                    "recorded_forward_ms": 1e3 * t_rec, "backward_ms": 1e3 * t_bwd,
                    "adjoint_over_forward": 1e3 * (t_rec + t_bwd) / ms_fwd,
                    "trajectory_states": 2 * nsteps,
                    "gradient_equals_checkpointed": bool(np.array_equal(gs, grads[prec][0])
                                                         and np.array_equal(ge, grads[prec][1]))}
        except Exception as e:  # reported, never fatal
            out[f"{prec}_whole_trajectory"] = {"unavailable": str(e)[:200]}
    gx, gex = grads["fp64_exact"][0], grads["fp64_exact"][1]
    gb, geb = grads["fp32_bulk"][0], grads["fp32_bulk"][1]
    out["bulk_forward_gradient_rel_l2"] = {
        "state": float(np.linalg.norm(gb - gx) / np.linalg.norm(gx)),
        "eta": float(np.linalg.norm(geb - gex) / np.linalg.norm(gex))}
    # central differences through the FP64 forward with the recorded dts
    dts = grads["fp64_exact"][2]
    rng = np.random.default_rng(2024)
    errs = []
    with Solver.from_setup(s, precision="fp64_exact", device=local_rank) as sol:
        def final_of(state, eta):
            sol.set_eta_table(eta)
            sol.set_state(state, apply_boundary=True)
            sol.run_fixed_dt(dts)
            return sol.get_state()

        for _ in range(ndirs):
            d = np.zeros_like(s.state)
            d[3:-3, 3:-3, 1:3] = rng.standard_normal(d[3:-3, 3:-3, 1:3].shape) * s.state[3:-3, 3:-3, 0:1]
            de = rng.standard_normal(s.eta_table.shape) * s.eta_table
            fd = _misfit_difference(final_of(s.state + h * d, s.eta_table + h * de),
                                    final_of(s.state - h * d, s.eta_table - h * de), target, fields) / (2 * h)
            ad = float((gx * d).sum() + (gex * de).sum())
            errs.append(abs(fd - ad) / max(abs(ad), 1e-300))
    errs = np.array(errs)
    out["fd_smooth_control"] = _fd_control(local_rank, h)
    out["fd_noisy_start"] = _fd_noisy_start(local_rank, s, target, fields)
    out["bulk_forward_gradient_vs_horizon"] = _bulk_gradient_vs_horizon(local_rank, s, target, fields)
    out["fd"] = {"h": h, "directions": ndirs, "forward": "fp64_exact",
                 "direction": "delta (rho vx, rho vy) of the initial state + delta eta, seeded normal",
                 "rel_err_median": float(np.median(errs)), "rel_err_max": float(errs.max()),
                 "frac_le_1e-6": float((errs <= 1e-6).mean()),
                 "note": "the Orszag-Tang start has exactly uniform rho and p, where minmod's slopes are 0 and "
                         "the step map is not differentiable, and 2000 steps of the vortex amplify an h = 1e-6 "
                         "perturbation out of the linear range; central differences then measure neither. "
                         "Against the oracle's dual-number tangent the adjoint agrees to 1e-10 "
                         "(tests/test_gpu_adjoint.py); fd_smooth_control is the same check where FD is valid"}
    return out


def _noisy(s, seed=6, amp=1e-3):
    """The adjoint workload's start with seeded relative noise on rho and on
    the thermal energy, so that no field is exactly uniform and minmod's
    slopes are nonzero (the step map is then differentiable there)."""
    import dataclasses

    import numpy as np

    rng = np.random.default_rng(seed)
    st = s.state.copy()
    core = st[3:-3, 3:-3]
    kin = 0.5 * (core[..., 1] ** 2 + core[..., 2] ** 2 + core[..., 3] ** 2) / core[..., 0]
    eth = core[..., 7] - kin - 0.5 * (core[..., 4] ** 2 + core[..., 5] ** 2 + core[..., 6] ** 2)
    f = 1.0 + amp * rng.uniform(-1.0, 1.0, core.shape[:2])
    g = 1.0 + amp * rng.uniform(-1.0, 1.0, core.shape[:2])
    core[..., 0] *= f
    core[..., 1:4] *= f[..., None]          # same velocity
    core[..., 7] = kin * f + eth * g        # same magnetic energy, thermal energy scaled by g
    return dataclasses.replace(s, state=st, name=s.name + "_noisy")


def _fd_noisy_start(local_rank, s0, target, fields, horizons=(20, 200), ndirs=32,
                    hs=(1e-4, 1e-6, 1e-8, 1e-9, 1e-10)):
    """Central differences and the Taylor remainder of the misfit against
    the FP64 adjoint on the adjoint workload's grid and eta field (512^2
    periodic Orszag-Tang, eta = 1e-3 exp(g/2)), from a start with rho and p
    noise, over horizons where an h-perturbation stays in the linear range.
    Per direction: the relative error of the central difference at each h
    and the best over h; the remainder |J(x + h d) - J(x) - h <grad, d>| at
    the h values, whose log-log slope is 2 where the map is smooth.

    Two kinds of direction: "field" perturbs (rho vx, rho vy) and eta in
    every cell; "local" perturbs them on a 3 x 3 patch.  The step map is
    piecewise smooth -- minmod switches between its arguments where two
    neighbouring differences are equal in size -- and a field direction
    crosses such kinks in many cells within any h, so its central
    differences converge only like a power of h below 1 (the field rows show
    it); a local direction reaches few cells and is where FD measures the
    gradient."""
    import numpy as np

    from resistivemhd_gpu_b200 import Solver

    s = _noisy(s0)
    out = {"workload": f"{s0.name} with 1e-3 rho and thermal-energy noise", "directions": ndirs, "h": list(hs),
           "forward": "fp64_exact", "direction": "delta (rho vx, rho vy) of the initial state + delta eta"}
    for nsteps in horizons:
        with Solver.from_setup(s, precision="fp64_exact", device=local_rank) as sol:
            sol.adjoint_forward(nsteps)
            final = sol.get_state()
            seed = np.zeros_like(final)
            seed[3:-3, 3:-3, fields] = final[3:-3, 3:-3, fields] - target[3:-3, 3:-3, fields]
            gs, ge = sol.adjoint_backward(seed)
            dts = sol.adjoint_dts()

            def final_of(state, eta):
                sol.set_eta_table(eta)
                sol.set_state(state, apply_boundary=True)
                sol.run_fixed_dt(dts)
                return sol.get_state()

            base = final_of(s.state, s.eta_table)
            for kind in ("local", "field"):
                rng = np.random.default_rng(11 + nsteps)
                best, per_h, slopes = [], {h: [] for h in hs}, []
                for _ in range(ndirs):
                    d = np.zeros_like(s.state)
                    de = np.zeros_like(s.eta_table)
                    if kind == "field":
                        d[3:-3, 3:-3, 1:3] = (rng.standard_normal(d[3:-3, 3:-3, 1:3].shape)
                                              * s.state[3:-3, 3:-3, 0:1])
                        de[...] = rng.standard_normal(s.eta_table.shape) * s.eta_table
                    else:
                        i0, j0 = rng.integers(3, s.nx - 6), rng.integers(3, s.ny - 6)
                        d[i0:i0 + 3, j0:j0 + 3, 1:3] = rng.standard_normal((3, 3, 2)) * s.state[i0:i0 + 3, j0:j0 + 3, 0:1]
                        de[i0:i0 + 3, j0:j0 + 3] = rng.standard_normal((3, 3)) * s.eta_table[i0:i0 + 3, j0:j0 + 3]
                    ad = float((gs * d).sum() + (ge * de).sum())
                    errs, rem = [], []
                    for h in hs:
                        fp = final_of(s.state + h * d, s.eta_table + h * de)
                        fm = final_of(s.state - h * d, s.eta_table - h * de)
                        fd = _misfit_difference(fp, fm, target, fields) / (2 * h)
                        e = abs(fd - ad) / max(abs(ad), 1e-300)
                        errs.append(e)
                        per_h[h].append(e)
                        rem.append(abs(_misfit_difference(fp, base, target, fields) - h * ad))
                    best.append(min(errs))
                    # slope of the remainder over the three largest h (above the rounding floor)
                    lr = np.log10(np.maximum(rem[:3], 1e-300))
                    slopes.append(float(np.polyfit(np.log10(hs[:3]), lr, 1)[0]))
                best = np.array(best)
                out[f"{kind}_steps_{nsteps}"] = {
                    "frac_le_1e-6": float((best <= 1e-6).mean()), "rel_err_median": float(np.median(best)),
                    "rel_err_max": float(best.max()),
                    "rel_err_median_per_h": {f"{h:g}": float(np.median(per_h[h])) for h in hs},
                    "taylor_remainder_slope_median": float(np.median(slopes)),
                    "taylor_remainder_slope_min": float(np.min(slopes))}
    return out


def _bulk_gradient_vs_horizon(local_rank, s, target, fields, horizons=(20, 200, 2000)):
    """Relative L2 distance of the gradients with the FP32-bulk forward from
    those with the FP64-exact forward (both reversed in FP64), by horizon: the
    FP32 trajectory departs from the FP64 one by its rounding, amplified by
    the flow, and the adjoint is linearised about it."""
    import numpy as np

    from resistivemhd_gpu_b200 import Solver

    out = {}
    for nsteps in horizons:
        g = {}
        for prec in ("fp32_bulk", "fp64_exact"):
            with Solver.from_setup(s, precision=prec, device=local_rank) as sol:
                sol.adjoint_forward(nsteps)
                final = sol.get_state()
                seed = np.zeros_like(final)
                seed[3:-3, 3:-3, fields] = final[3:-3, 3:-3, fields] - target[3:-3, 3:-3, fields]
                g[prec] = sol.adjoint_backward(seed)
        gx, gex = g["fp64_exact"]
        gb, geb = g["fp32_bulk"]
        out[f"steps_{nsteps}"] = {"state": float(np.linalg.norm(gb - gx) / np.linalg.norm(gx)),
                                  "eta": float(np.linalg.norm(geb - gex) / np.linalg.norm(gex))}
    return out


def _fd_control(local_rank, h, n=128, nsteps=20, ndirs=16):
    """Central differences against the adjoint on a generic smooth periodic
    state (no exactly uniform fields, a horizon within the linear range),
    along directions on a 3 x 3 patch; each direction takes the better of h
    and h/10, since a limiter kink within h of the base point spoils the
    quotient of that h only."""
    import numpy as np

    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(n, n, seed=3, bc="periodic", with_table=True)
    target = s.state.copy()
    fields = [0, 4, 5, 6]

    with Solver.from_setup(s, precision="fp64_exact", device=local_rank) as sol:
        sol.adjoint_forward(nsteps)
        final = sol.get_state()
        seed = np.zeros_like(final)
        seed[3:-3, 3:-3, fields] = final[3:-3, 3:-3, fields] - target[3:-3, 3:-3, fields]
        gs, ge = sol.adjoint_backward(seed)
        dts = sol.adjoint_dts()

        def final_of(state, eta):
            sol.set_eta_table(eta)
            sol.set_state(state, apply_boundary=True)
            sol.run_fixed_dt(dts)
            return sol.get_state()

        rng = np.random.default_rng(7)
        errs = []
        for _ in range(ndirs):
            d = np.zeros_like(s.state)
            de = np.zeros_like(s.eta_table)
            i0, j0 = rng.integers(3, s.nx - 6), rng.integers(3, s.ny - 6)
            d[i0:i0 + 3, j0:j0 + 3, 1:3] = rng.standard_normal((3, 3, 2))
            de[i0:i0 + 3, j0:j0 + 3] = rng.standard_normal((3, 3)) * s.eta_table[i0:i0 + 3, j0:j0 + 3]
            ad = float((gs * d).sum() + (ge * de).sum())
            e = []
            for hh in (h, h / 10):
                fd = _misfit_difference(final_of(s.state + hh * d, s.eta_table + hh * de),
                                        final_of(s.state - hh * d, s.eta_table - hh * de), target, fields) / (2 * hh)
                e.append(abs(fd - ad) / max(abs(ad), 1e-300))
            errs.append(min(e))
    errs = np.array(errs)
    return {"workload": f"random_smooth_{n}x{n}_{nsteps}steps", "directions": ndirs, "h": [h, h / 10],
            "rel_err_median": float(np.median(errs)), "rel_err_max": float(errs.max()),
            "frac_le_1e-6": float((errs <= 1e-6).mean())}


def contact_block(args, setup, label, local_rank):
    """The CT-Contact step on the headline workload, against the
    stage-1-EMF step in the same arithmetic (FP64 without contraction)."""
    import dataclasses

    from resistivemhd_gpu_b200 import Solver

    out = {"workload": label, "steps": args.steps}
    for ct in ("stage1", "contact"):
        s = dataclasses.replace(setup, ct=ct)
        with Solver.from_setup(s, precision="fp64_exact", device=local_rank) as sol:
            if ct == "stage1":
                sol.autotune(4)
            sol.run(args.warmup)
            ms = sol.run_timed(args.steps)
            out[ct] = {"value": setup.interior_cells * args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps,
                       "crashed": sol.check_crashed()}
    out["contact_over_stage1_time"] = out["contact"]["ms_per_step"] / out["stage1"]["ms_per_step"]
    out["note"] = ("CT-Contact runs as 13 launches per step (tiled fluxes to HBM, per-cell EMF inputs, the "
                   "corner EMFs, one CT at the end); the stage-1-EMF step is the fused 4-launch pipeline")
    return out


def _shard(setups_list, world):
    """Greedy largest-first assignment of runs to ranks by cell count."""
    order = sorted(range(len(setups_list)), key=lambda r: -setups_list[r].interior_cells)
    load = [0] * world
    parts = [[] for _ in range(world)]
    for r in order:
        w = min(range(world), key=lambda q: load[q])
        parts[w].append(r)
        load[w] += setups_list[r].interior_cells
    return [sorted(p) for p in parts]


def ensemble_block(args, rank, world, local_rank, dist, nsteps=500, nruns=256):
    """Batched ensemble in FP32-bulk against the FP64 path looped run by run."""
    import torch

    from resistivemhd_gpu_b200 import Batch, Solver, setups

    runs = setups.ensemble(nruns)
    mine = _shard(runs, world)[rank]
    total_cells = sum(r.interior_cells for r in runs)
    out = {"runs": nruns, "steps": nsteps, "cells": total_cells, "sizes": list(setups.ENSEMBLE_SIZES),
           "eta": "log-uniform [1e-4, 1e-2]", "kinds": "Orszag-Tang (even) / Kelvin-Helmholtz (odd)",
           "sharding": f"{world} rank(s), largest-first by cells, no collective on the data path"}
    my_sets = [runs[r] for r in mine]
    with Batch(my_sets, precision="fp32_bulk", device=local_rank) as b:
        shape, ctas = b.autotune(trial_steps=4)
        table = b.tuning()
        default_ms = next((m for sh, c, m in table if (sh, c) == (0, 2)), None)
        best_ms = min(m for _, _, m in table)
        out["autotune"] = {"chosen": [shape, ctas], "points": [{"shape": sh, "ctas_per_sm": c, "ms_per_step": m}
                                                               for sh, c, m in table],
                           "default": [0, 2],
                           "margin_over_default": None if not default_ms else default_ms / best_ms - 1.0}
        b.run(3)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ms = b.run_timed(nsteps)
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        out["batch_fp32_bulk"] = {"value": total_cells * nsteps / (ms * 1e-3), "ms": ms, "launch": [shape, ctas]}
        bulk_final = {r: b[q].get_state() for q, r in enumerate(mine)} if world == 1 else None
        bulk_time = {r: b[q].total_time for q, r in enumerate(mine)} if world == 1 else None
    if world > 1:
        return out
    # the FP64 drop-in path, one run at a time
    ms_loop = 0.0
    errs, tdiff = [], []
    for r, s in enumerate(runs):
        with Solver.from_setup(s, precision="fp64_exact", device=local_rank) as sol:
            sol.run(3)
            sol.set_state(s.state, apply_boundary=True)      # total_time is not reset (nor is the reference's)
            t_start = sol.total_time
            ms_loop += sol.run_timed(nsteps + 3)
            elapsed = sol.total_time - t_start
            ref = _diagnostics(sol.get_state(), s.dx, s.dy, s.gamma)
            got = _diagnostics(bulk_final[r], s.dx, s.dy, s.gamma)
            errs.append(max(_rel_l1(got[k], ref[k]) for k in ("rho", "p", "B")))
            tdiff.append(abs(bulk_time[r] - elapsed) / elapsed)
    loop_value = total_cells * (nsteps + 3) / (ms_loop * 1e-3)
    out["loop_fp64_exact"] = {"value": loop_value, "ms_per_500_steps": ms_loop * nsteps / (nsteps + 3)}
    out["speedup_vs_loop_fp64"] = out["batch_fp32_bulk"]["value"] / loop_value
    out["bulk_vs_fp64_max_rel_l1"] = float(max(errs))
    out["bulk_vs_fp64_total_time_max_rel_diff"] = float(max(tdiff))
    out["note"] = ("rel L1 of rho, p, B after 503 steps (3 warm-up + 500), each run with its own CFL dt, "
                   "so it includes the small difference in elapsed time")
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64_fast", "fp64_exact", "fp32_bulk"], default="fp64_exact")
    ap.add_argument("--workload", choices=["harris", "orszag_tang"], default="harris")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-baselines", dest="baselines", action="store_false")
    ap.add_argument("--no-precision", dest="precision_block", action="store_false")
    ap.add_argument("--no-adjoint", dest="adjoint_block", action="store_false")
    ap.add_argument("--no-contact", dest="contact_block", action="store_false")
    ap.add_argument("--no-ensemble", dest="ensemble_block", action="store_false")
    ap.add_argument("--quick", action="store_true", help="headline only (no extra blocks, baselines or e2e)")
    ap.add_argument("--tile-shapes", type=int, nargs=2, metavar=("STAGE1", "STAGE2"), default=None,
                    help="the stage kernels' tile shapes instead of the autotuner's pick")
    ap.add_argument("--study", choices=sorted(STUDIES), default=None,
                    help="instead of the benchmark: the long FP32-bulk / FP64 error study of one workload")
    ap.add_argument("--study-steps", type=int, default=0, help="override the study's step count")
    args = ap.parse_args()
    if args.quick:
        args.precision_block = args.adjoint_block = args.ensemble_block = args.contact_block = False
        args.baselines = args.e2e = False
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.study:
        if rank == 0:
            print(json.dumps(precision_study(args, local_rank)), flush=True)
        return

    import torch

    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        ours_arm(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
