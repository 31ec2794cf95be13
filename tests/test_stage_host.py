"""The fused stage kernel on the CPU: the exact variant (stage_exact.cu) and
the ghost-fill / CFL kernels compiled for the host (tests/host_build.py,
RMHD_HOST_EMULATION with tests/host_tma.cpp for the tile staging; the
kernels run one host thread per CUDA thread) and driven as enqueue_step
drives them (tests/stage_host.cpp).  Built without contraction, as nvcc
builds the exact variant (-fmad=false), states and dts must equal the
oracle's bit for bit, as tests/test_gpu_parity.py requires of the CUDA run.
Shared memory starts each block as NaN bytes, so a read of a word the
kernel did not stage or compute would show in the results."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from host_build import compile_unit, link, shim_dir

HERE = Path(__file__).resolve().parent
BC = {"periodic": 0, "symmetric": 1, "zero_gradient": 2, "wall": 3, "flare": 4}
EMU = "-DRMHD_HOST_EMULATION"


# the host flags that model each variant's device build: -fmad=false for the
# exact one, contraction into fused multiply-adds for the others
VARIANTS = {"exact": ("stage_exact.cu", ["-ffp-contract=off"]),
            "fast": ("stage_fast.cu", ["-ffp-contract=fast", "-mfma"]),
            "bulk32": ("stage_bulk32.cu", ["-ffp-contract=fast", "-mfma"])}


def build_stage(d: Path, extra: tuple[str, ...] = (), variant: str = "exact"):
    """A stage kernel variant, aux_kernels.cu, the staging emulation and the
    step driver as a host library; `extra` adds compiler flags to every
    unit."""
    shim_dir(d)
    unit, flags = VARIANTS[variant]
    objs = [compile_unit(d, unit, [*flags, EMU, *extra],
                         threaded=("stage_kernel", "stage_batch_kernel"), headers=("stage_impl.cuh",)),
            compile_unit(d, "aux_kernels.cu", ["-ffp-contract=off", *extra],
                         threaded=("kernel", "rate_kernel", "boundary_batch_kernel"))]
    lib = link(d, objs, [HERE / "host_tma.cpp", HERE / "stage_host.cpp"], "libstagehost.so",
               (EMU, f"-DSTAGE_VARIANT={variant}", *extra))
    D = ctypes.POINTER(ctypes.c_double)
    lib.host_stage_run.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 + [
        ctypes.c_int, ctypes.c_int, D, ctypes.c_int, D, ctypes.c_int, D, ctypes.c_int, D]
    lib.host_stage_run.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="module")
def host_stage(tmp_path_factory):
    return build_stage(tmp_path_factory.mktemp("stagehost"))


def run_host(lib, s, nsteps, shape, apply_boundary=True, fixed_dts=None):
    D = ctypes.POINTER(ctypes.c_double)
    tab = None if s.eta_table is None else np.ascontiguousarray(s.eta_table, dtype=np.float64)
    state = np.ascontiguousarray(s.state, dtype=np.float64).copy()
    dts = np.zeros(max(nsteps, 1))
    fixed = None if fixed_dts is None else np.ascontiguousarray(fixed_dts, dtype=np.float64)
    rc = lib.host_stage_run(s.nx, s.ny, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta, BC[s.bc],
                            BC[s.bc_y] if s.bc_y else -1, None if tab is None else tab.ctypes.data_as(D), shape,
                            state.ctypes.data_as(D), nsteps, dts.ctypes.data_as(D), int(apply_boundary),
                            None if fixed is None else fixed.ctypes.data_as(D))
    assert rc != -1, "a tile's staging wait expired"
    return state, dts[:nsteps], rc - 1 if rc > 0 else -1


@pytest.mark.parametrize("shape", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("dims,nsteps,bc,bc_y,with_table", [
    ((20, 18), 3, "periodic", None, False),
    ((37, 29), 2, "periodic", None, True),
    ((26, 40), 2, "symmetric", None, True),
    ((23, 19), 2, "periodic", "symmetric", False),
    ((21, 25), 2, "flare", "wall", True),
    ((18, 17), 2, "zero_gradient", "periodic", False),
])
def test_host_stage_step_equals_oracle(host_stage, oracle, shape, dims, nsteps, bc, bc_y, with_table):
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(*dims, seed=17, bc=bc, bc_y=bc_y, with_table=with_table)
    want, want_dts, want_crash = oracle.run(s, s.state, nsteps)
    got, got_dts, got_crash = run_host(host_stage, s, nsteps, shape)
    assert got_crash == want_crash
    assert np.array_equal(got_dts, want_dts)
    assert np.array_equal(got, want, equal_nan=True)


@pytest.mark.parametrize("shape,ctas", [(0, 1), (0, 3), (1, 2), (2, 1), (3, 1), (4, 2), (5, 3)])
def test_host_batch_equals_single_oracle_runs(host_stage, oracle, shape, ctas):
    """The persistent batch kernel over runs of uneven size and walls: a few
    CTAs walk the tile table (flipping the mbarrier's phase tile by tile),
    and every run equals its own oracle run bit for bit."""
    from resistivemhd_gpu_b200 import setups

    setups_ = [setups.random_smooth_state(21, 14, seed=31, bc="periodic"),
               setups.random_smooth_state(9, 27, seed=32, bc="symmetric"),
               setups.random_smooth_state(16, 16, seed=33, bc="periodic", bc_y="symmetric")]
    nsteps = 2
    I = lambda v: (ctypes.c_int * len(v))(*v)          # noqa: E731
    F = lambda v: (ctypes.c_double * len(v))(*v)       # noqa: E731
    states = np.concatenate([s.state.ravel() for s in setups_])
    dts = np.zeros(len(setups_) * nsteps)
    lib = host_stage
    lib.host_batch_run.restype = ctypes.c_int
    D = ctypes.POINTER(ctypes.c_double)
    rc = lib.host_batch_run(len(setups_), I([s.nx for s in setups_]), I([s.ny for s in setups_]),
                            F([s.dx for s in setups_]), F([s.dy for s in setups_]), F([s.eta for s in setups_]),
                            I([BC[s.bc] for s in setups_]), I([BC[s.bc_y] if s.bc_y else -1 for s in setups_]),
                            ctypes.c_double(setups_[0].gamma), ctypes.c_double(setups_[0].cfl),
                            ctypes.c_double(setups_[0].eps), shape, ctas, states.ctypes.data_as(D), nsteps,
                            dts.ctypes.data_as(D))
    assert rc == 0
    off = 0
    for r, s in enumerate(setups_):
        n = s.state.size
        want, want_dts, _ = oracle.run(s, s.state, nsteps)
        assert np.array_equal(states[off:off + n].reshape(s.state.shape), want, equal_nan=True), r
        assert np.array_equal(dts[r * nsteps:(r + 1) * nsteps], want_dts), r
        off += n


@pytest.fixture(scope="module", params=["fast", "bulk32"])
def host_stage_contracted(request, tmp_path_factory):
    if " fma " not in open("/proc/cpuinfo").read().replace("\n", " "):
        pytest.skip("the host has no fused multiply-add to model the device build with")
    return request.param, build_stage(tmp_path_factory.mktemp("stagehost_" + request.param), variant=request.param)


# relative L1 per field against the exact oracle after the steps (the GPU
# tests' bounds: fp64_fast differs by rounding only, fp32_bulk by its FP32 core)
HOST_REL_L1 = {"fast": 1e-12, "bulk32": 1e-5}


@pytest.mark.parametrize("shape", [0, 1, 3, 4, 5])
@pytest.mark.parametrize("dims,bc,bc_y,with_table", [
    ((37, 29), "periodic", None, True),
    ((26, 40), "symmetric", None, True),
    ((21, 25), "flare", "wall", False),
])
def test_host_contracted_variants_within_bounds(host_stage_contracted, oracle, shape, dims, bc, bc_y, with_table):
    """The fast and FP32-bulk variants built as nvcc builds them (contracted;
    the hardware reciprocal and square-root seeds replaced by correctly
    rounded values) stay within their bounds of the exact oracle."""
    from resistivemhd_gpu_b200 import setups

    variant, lib = host_stage_contracted
    s = setups.random_smooth_state(*dims, seed=19, bc=bc, bc_y=bc_y, with_table=with_table)
    want, want_dts, _ = oracle.run(s, s.state, 3)
    got, got_dts, crashed = run_host(lib, s, 3, shape)
    assert crashed == -1 and np.isfinite(got).all()
    assert np.allclose(got_dts, want_dts, rtol=HOST_REL_L1[variant], atol=0)
    for f in range(8):
        rel = np.abs(got[..., f] - want[..., f]).sum() / max(np.abs(want[..., f]).sum(), 1e-300)
        assert rel <= HOST_REL_L1[variant], (variant, f, rel)


@pytest.mark.parametrize("shape", [0, 1])
def test_host_stage_matches_reference_golden_outputs(host_stage, shape):
    """The exact variant's host build against the committed outputs of the
    reference library itself (tests/golden, from the reference built for the
    host): states, dts and the total time, bit for bit."""
    from conftest import GOLDEN_CASES, load_golden

    assert GOLDEN_CASES
    for name in GOLDEN_CASES:
        s, init, final, dts, total_time = load_golden(name)
        s.state = init
        got, got_dts, crashed = run_host(host_stage, s, len(dts), shape)
        assert crashed == -1, name
        assert np.array_equal(got_dts, dts), name
        assert np.array_equal(got, final), name


def test_host_exact_reproduces_the_reference_nan_at_the_degenerate_face(host_stage):
    """The plasmoid sheet's degenerate HLLD face (tests/test_degenerate_face.py):
    one fixed-dt step of the window, no boundary first; the exact variant's
    host build turns the same three cells non-finite as the reference's
    arithmetic, and equals the oracle bit for bit at the centre."""
    import test_degenerate_face as F

    s, dt, bad = F._window()
    want, _ = F._oracle_step()
    got, _, _ = run_host(host_stage, s, 1, 0, apply_boundary=False, fixed_dts=[dt])
    assert np.array_equal(got[F.CENTRE], want[F.CENTRE], equal_nan=True)
    assert sorted(map(tuple, np.argwhere(~np.isfinite(got[..., 7])).tolist())) == sorted(bad)


def test_host_contracted_variants_survive_the_degenerate_face(host_stage_contracted):
    import test_degenerate_face as F

    variant, lib = host_stage_contracted
    s, dt, _ = F._window()
    got, _, crashed = run_host(lib, s, 1, 0, apply_boundary=False, fixed_dts=[dt])
    c = got[F.CENTRE]
    assert crashed == -1 and np.isfinite(c).all(), variant
    rel = np.abs(c[..., 7] - s.state[F.CENTRE][..., 7]) / np.abs(s.state[F.CENTRE][..., 7])
    assert rel.max() < 1e-2, (variant, rel.max())


def test_host_contracted_variants_take_the_nan_path(host_stage_contracted, oracle):
    """A NaN energy makes the wave speeds of the interfaces around it NaN.
    The contracted variants' common-case flux declines those interfaces, and
    the pass after the flux loop forms them as NaN fluxes, as the reference's
    weighted sum does: after one step the same cells are non-finite as in
    the oracle's run, and the crash flag is raised."""
    from resistivemhd_gpu_b200 import setups

    variant, lib = host_stage_contracted
    s = setups.random_smooth_state(40, 36, seed=11, bc="periodic")
    st = s.state.copy()
    st[18, 15, 7] = np.nan
    s.state = st
    want, _, crashed_at = oracle.run(s, st, 1)
    got, _, crashed = run_host(lib, s, 1, 4)
    assert crashed_at == 0 and crashed == 0, variant
    assert np.array_equal(~np.isfinite(got), ~np.isfinite(want)), variant
