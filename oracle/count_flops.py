"""Floating-point operations per interior cell-update of the step, counted by
running the oracle's templated restatement (rmhd2d_tangent.cpp) on its
operation-counting scalar: the algorithm's operation count as the reference
evaluates it (every HLLD candidate formed and weighted, IEEE divisions and
square roots), over the whole array including ghost cells, divided by the
interior cells.  TEST INFRASTRUCTURE: the number feeds the FP64 roofline in
profiles/; the product never runs this.

    python oracle/count_flops.py [--workload harris] [--steps 1]
"""
import argparse
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def main() -> None:
    from oracle.oracle import OracleLib, TangentLib
    from resistivemhd_gpu_b200 import setups

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["harris", "orszag_tang"], default="harris")
    ap.add_argument("--steps", type=int, default=1)
    args = ap.parse_args()
    s = setups.harris_sheet(2048, 1024) if args.workload == "harris" else setups.orszag_tang(256)
    _, dts, _ = OracleLib().run(s, s.state, args.steps)
    _, c = TangentLib().count_ops(s, s.state, dts)
    n = s.interior_cells * args.steps
    flops = c["add"] + c["mul"] + c["div"] + c["sqrt"]
    print(json.dumps({"workload": args.workload, "steps": args.steps, "counts": c,
                      "per_cell_update": {k: v / n for k, v in c.items()}, "flops_per_cell_update": flops / n}))


if __name__ == "__main__":
    main()
