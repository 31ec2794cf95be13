"""The whole C ABI on the CPU: every unit of resistivemhd_gpu_b200/csrc built
for the host (tests/host_build.py; the runtime calls of api.cu answered by
tests/cuda_host_runtime.h, with graph capture recorded and replayed) into
one library, which this module hands to the Python mirror in place of
librmhd2d.so for its own tests only.  The GPU tests' own functions then run
on it: the drop-in's parity through the graph-replayed run and step paths,
the checkpoint-interval and whole-trajectory invariances of the adjoint, its
refusals, batches, snapshots, walls and the CT-Contact step.  The product never loads this library."""
import numpy as np
import pytest

from host_build import build_host_abi, has_fma


@pytest.fixture(scope="module")
def host_abi(tmp_path_factory):
    if not has_fma():
        pytest.skip("the host has no fused multiply-add to model the device build with")
    return build_host_abi(tmp_path_factory.mktemp("abihost"))


@pytest.fixture
def on_host(host_abi, monkeypatch):
    """The Python mirror bound to the host build for one test."""
    from resistivemhd_gpu_b200 import _lib

    monkeypatch.setattr(_lib, "_lib", host_abi)
    return host_abi


def test_host_abi_step_and_run_paths_equal_oracle(on_host, oracle):
    """rmhd2d_run (two-step graphs), rmhd2d_step_rk2 (one-step graphs) and a
    frozen-dt run all give the oracle's states and dts bit for bit."""
    from resistivemhd_gpu_b200 import Solver, setups

    s = setups.random_smooth_state(21, 17, seed=41, bc="symmetric", with_table=True)
    want, want_dts, _ = oracle.run(s, s.state, 5)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        sol.run(3)
        sol.step()
        sol.step()
        assert np.array_equal(sol.get_state(), want)
        assert sol.dt == want_dts[-1]
        assert sol.total_time == pytest.approx(want_dts.sum(), rel=1e-15)
        sol.set_state(s.state, apply_boundary=True)
        sol.run_fixed_dt(want_dts)
        assert np.array_equal(sol.get_state(), want)
        sol.step()                                  # back on the CFL dt after the frozen run
        assert sol.dt == oracle.calc_dt(s, want)


def test_host_abi_gpu_adjoint_tests(on_host, oracle, tangent):
    """tests/test_gpu_adjoint.py's invariance and refusal tests, and its
    tangent test with the whole trajectory kept, on the host build."""
    import test_gpu_adjoint as G

    G.test_checkpoint_interval_changes_nothing_and_state_is_restored(None)
    G.test_adjoint_needs_a_recorded_run(None)
    G.test_adjoint_rejects_other_walls(None)
    G.test_adjoint_matches_oracle_tangent(None, oracle, tangent, True, (22, 19), 5, -1, "symmetric", None)
    G.test_adjoint_matches_oracle_tangent(None, oracle, tangent, False, (20, 18), 5, 2, "periodic", None)
    G.test_adjoint_on_the_harris_sheet(None, tangent)


def test_host_abi_gpu_batch_tests(on_host):
    import test_gpu_batch as B

    B.test_batch_odd_steps_and_graph_replay(None)
    B.test_member_cannot_step_alone(None)
    # (the batch and solver autotuners run in tests/host_sanitized_run.py)


def test_host_abi_gpu_parity_and_io_tests(on_host, oracle, tmp_path):
    """tests/test_gpu_parity.py's graph/step, dt, snapshot, crash-flag,
    reference-mirror and extreme-value tests, tests/test_walls.py's wall
    pairings with both CT schemes, and tests/test_gpu_contact.py's refusals,
    on the host build."""
    import test_gpu_contact as C
    import test_gpu_parity as P
    import test_walls as W

    P.test_run_graph_equals_step_loop(None)
    P.test_calculate_dt_matches_oracle(None, oracle)
    P.test_save_load_resume(None, tmp_path)
    P.test_crash_flag_on_host_injected_nan(None)
    P.test_reference_class_mirror(None, oracle)
    for case in ("huge", "nan"):
        P.test_exact_bitwise_vs_oracle_on_extreme_values(None, oracle, case)
    for bcx, bcy in (("flare", "wall"), ("zero_gradient", "symmetric")):
        for ct in ("stage1", "contact"):
            W.test_walls_match_oracle_bit_for_bit(None, oracle, bcx, bcy, ct)
    C.test_contact_refuses_batch_adjoint_and_profile(None)


def test_host_abi_smoke(on_host, capsys):
    """__graft_entry__.smoke(), run against the host build."""
    import __graft_entry__ as entry

    entry.smoke()
    assert "smoke ok" in capsys.readouterr().out
