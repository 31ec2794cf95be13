"""TEST INFRASTRUCTURE, run by tests/test_host_memory_safety.py in a child
process with the address sanitizer's runtime preloaded.  The whole C ABI
(every unit of resistivemhd_gpu_b200/csrc, api.cu included) is built for the
host with -fsanitize=address,undefined (tests/host_build.py) and driven
through the Python mirror: every wall pairing of the stage-1-EMF step (in
all three precisions on the diagonal pairings) and half of them with the
CT-Contact step, on small ragged grids down to the smallest legal 6 x 6
interior, the adjoint with checkpoints and with the
whole trajectory kept on every periodic/symmetric pairing, a batch, and the
batch and solver autotuners.  Any read or write outside an allocation, and any undefined
behaviour, aborts the child: the kernels' index arithmetic and the ABI's
buffer handling are checked against their buffers on the CPU.  Each exact
run is also compared with the oracle.  Prints "ok" at the end."""
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))

from host_build import SANITIZE, build_host_abi  # noqa: E402

X_WALLS = ("periodic", "symmetric", "zero_gradient", "flare")
Y_WALLS = ("periodic", "symmetric", "zero_gradient", "wall")


def main() -> None:
    from oracle.oracle import OracleLib
    from resistivemhd_gpu_b200 import Batch, Solver, _lib, setups

    oracle = OracleLib()
    _lib._lib = build_host_abi(Path(tempfile.mkdtemp()), tuple(SANITIZE))

    for k, bcx in enumerate(X_WALLS):
        for m, bcy in enumerate(Y_WALLS):
            dims = [(6, 6), (6, 7), (9, 6), (13, 11)][(k + m) % 4]
            s = setups.random_smooth_state(*dims, seed=3 + k + m, bc=bcx, bc_y=bcy, with_table=(k + m) % 2 == 0)
            # every pairing in FP64-exact; the contracted variants on the
            # diagonal, CT-Contact on every other pairing
            for ct in ("stage1", "contact") if (k + m) % 2 == 0 else ("stage1",):
                s.ct = ct
                want, want_dts, crashed = oracle.run(s, s.state, 2)
                extra = ("fp64_fast", "fp32_bulk") if ct == "stage1" and k == m else ()
                for precision in ("fp64_exact", *extra):
                    with Solver.from_setup(s, precision=precision) as sol:
                        sol.run(2)
                        got = sol.get_state()
                    # (the oracle stops at a crash, as the reference's drivers do; the
                    # smallest symmetric boxes crash in the reference's arithmetic)
                    if precision == "fp64_exact" and crashed < 0:
                        assert np.array_equal(got, want, equal_nan=True), (bcx, bcy, ct)
            s.ct = "stage1"

    w_rng = np.random.default_rng(2)
    for bcx in ("periodic", "symmetric"):
        for bcy in ("periodic", "symmetric"):
            s = setups.random_smooth_state(20, 18, seed=21, bc=bcx, bc_y=bcy, with_table=True)
            w = w_rng.standard_normal(s.state.shape)
            with Solver.from_setup(s, precision="fp64_exact") as sol:
                grads = []
                for interval in (1, -1):
                    sol.set_state(s.state, apply_boundary=True)
                    sol.adjoint_forward(2, interval)
                    grads.append(sol.adjoint_backward(w))
                sol.adjoint_release()
            assert all(np.array_equal(g[0], grads[0][0]) and np.array_equal(g[1], grads[0][1]) for g in grads), \
                (bcx, bcy)

    with Batch([setups.random_smooth_state(9, 14, seed=8), setups.random_smooth_state(15, 7, seed=9)]) as b:
        b.run(3)
        b.autotune(2)
    with Solver.from_setup(setups.random_smooth_state(10, 9, seed=10)) as sol:
        sol.autotune(2)
    print("ok", flush=True)


if __name__ == "__main__":
    main()
