"""TEST INFRASTRUCTURE, run by tests/test_host_memory_safety.py in a child
process with the address sanitizer's runtime preloaded.  The host builds of
the fused stage kernel (stage_exact.cu), the adjoint kernels (adjoint.cu,
adjoint_prep.cu), the CT-Contact kernels (contact.cu), the ghost fill and CFL reduction (aux_kernels.cu) and the
allocation-free dt (noalloc_dt.cu) are compiled with
-fsanitize=address,undefined and run on small ragged grids, down to the
smallest legal 6 x 6 interior, with every wall pairing they support; then
the whole C ABI, api.cu included, built the same way, steps, runs the
adjoint and a batch.  Any
read or write outside an allocation, and any undefined behaviour, aborts
the child: the kernels' index arithmetic is checked against their buffers on
the CPU.  Prints "ok" at the end."""
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent))

from host_build import SANITIZE  # noqa: E402


def main() -> None:
    import test_adjoint_host as A
    import test_contact_host as C
    from oracle.oracle import OracleLib
    from resistivemhd_gpu_b200 import setups

    import test_aux_host as X
    import test_stage_host as S
    from concurrent.futures import ThreadPoolExecutor

    from host_build import build_host_abi

    oracle = OracleLib()
    tmp = Path(tempfile.mkdtemp())
    for sub in ("adj", "ct", "aux", "stage", "abi"):
        (tmp / sub).mkdir()
    san = tuple(SANITIZE)
    # the five sanitized builds at once (each is compiler subprocesses)
    with ThreadPoolExecutor(max_workers=5) as pool:
        futures = [pool.submit(A._build, tmp / "adj", False, san), pool.submit(C.build_contact, tmp / "ct", san),
                   pool.submit(X.build_aux, tmp / "aux", san), pool.submit(S.build_stage, tmp / "stage", san),
                   pool.submit(build_host_abi, tmp / "abi", san)]
        adj, ct, aux, stage, abi = [f.result() for f in futures]
    for shape, bc, bc_y, table in [((13, 11), "periodic", None, True), ((12, 15), "symmetric", None, False),
                                   ((14, 12), "periodic", "symmetric", True), ((11, 13), "symmetric", "periodic", False),
                                   ((6, 6), "periodic", None, True), ((6, 7), "symmetric", None, False),
                                   ((7, 6), "periodic", "symmetric", False)]:
        s = setups.random_smooth_state(*shape, seed=3, bc=bc, bc_y=bc_y, with_table=table)
        _, dts, crashed, un, us = oracle.run_keep_stages(s, s.state, 2)
        # the smallest symmetric boxes crash in the reference's arithmetic;
        # their trajectory up to and including the crashing step still runs
        n = 2 if crashed < 0 else crashed + 1
        gs, ge = A.backward(adj, s, un[:n], us[:n], dts[:n], np.random.default_rng(1).standard_normal(s.state.shape))
        if crashed < 0:
            assert np.isfinite(gs).all() and np.isfinite(ge).all()
    for shape, bc, bc_y, table in [((13, 11), "periodic", None, True), ((12, 15), "symmetric", None, False),
                                   ((14, 12), "flare", "wall", True), ((11, 13), "zero_gradient", "periodic", False),
                                   ((6, 6), "periodic", None, False), ((6, 7), "symmetric", "wall", True)]:
        s = setups.random_smooth_state(*shape, seed=3, bc=bc, bc_y=bc_y, with_table=table)
        s.ct = "contact"
        want, want_dts, _ = oracle.run(s, s.state, 2)
        got, got_dts, _ = C.run_host(ct, s, 2)
        assert np.array_equal(got, want, equal_nan=True) and np.array_equal(got_dts, want_dts)
    for bcx in ("periodic", "symmetric", "zero_gradient", "flare"):
        for bcy in ("periodic", "symmetric", "zero_gradient", "wall"):
            s = setups.random_smooth_state(6, 7, seed=4, bc=bcx, bc_y=bcy)
            got, dt, _, _ = X.set_state_dt(aux, s, s.state, ghost_rates=True)
            assert np.array_equal(got, oracle.boundary(s, s.state), equal_nan=True)
            assert X.same(X.dt_noalloc(aux, s, got), dt)
    for shape in (0, 1):
        for dims, bc, bc_y, table in [((6, 6), "periodic", None, True), ((19, 13), "symmetric", None, False),
                                      ((9, 7), "flare", "wall", True), ((14, 11), "periodic", "symmetric", False)]:
            s = setups.random_smooth_state(*dims, seed=5, bc=bc, bc_y=bc_y, with_table=table)
            want, want_dts, _ = oracle.run(s, s.state, 1)
            got, got_dts, _ = S.run_host(stage, s, 1, shape)
            assert np.array_equal(got, want, equal_nan=True) and np.array_equal(got_dts, want_dts, equal_nan=True)
    # the C ABI's host code (api.cu) over the same kernels: stepping through
    # its graph paths, the adjoint with checkpoints and with the whole
    # trajectory kept, a batch, snapshots of errors
    from resistivemhd_gpu_b200 import Batch, Solver, _lib

    _lib._lib = abi
    s = setups.random_smooth_state(13, 11, seed=7, bc="symmetric", with_table=True)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.run(3)
        sol.step()
        sol.calculate_dt()
        w = np.random.default_rng(2).standard_normal(s.state.shape)
        for interval in (0, 2, -1):
            sol.set_state(s.state, apply_boundary=True)
            sol.adjoint_forward(4, interval)
            sol.adjoint_backward(w)
        sol.adjoint_release()
    for precision in ("fp64_fast", "fp32_bulk"):
        with Solver.from_setup(s, precision=precision) as sol:
            sol.run(2)
    with Batch([setups.random_smooth_state(9, 14, seed=8), setups.random_smooth_state(15, 7, seed=9)]) as b:
        b.run(3)
        b.autotune(2)
    print("ok", flush=True)


if __name__ == "__main__":
    main()
