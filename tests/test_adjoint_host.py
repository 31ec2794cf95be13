"""The discrete adjoint's kernels on the CPU: adjoint.cu and adjoint_prep.cu
compiled for the host (tests/cuda_host_shim.h, each kernel launch rewritten
into a loop over its blocks and threads) and driven by the reverse loop of
rmhd2d_adjoint_backward (tests/adjoint_host.cpp) over the oracle's forward
trajectory.  The gradient is checked against the oracle's dual-number
tangent as the GPU tests check the CUDA run (tests/test_gpu_adjoint.py), so
changes to the adjoint's arithmetic, transposes and stage wiring are caught
without a GPU."""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from host_build import compile_unit, link, rewrite_launches, shim_dir

HERE = Path(__file__).resolve().parent
ADJ_REL = 1e-10


def _build(d: Path, contracted: bool, extra: tuple[str, ...] = ()):
    """The adjoint kernels and the reverse loop as a host library.  With
    `contracted`, adjoint.cu is built the way nvcc builds it for the device
    (fused multiply-add wherever the compiler finds one; the explicitly
    rounded operations kept apart, RMHD_ADJ_HOST_RN) and adjoint_prep.cu
    without contraction (-fmad=false on the device)."""
    shim_dir(d)
    objs = [compile_unit(d, "adjoint.cu", [*(["-ffp-contract=fast", "-mfma", "-DRMHD_ADJ_HOST_RN"] if contracted
                                            else ["-ffp-contract=off"]), *extra]),
            compile_unit(d, "adjoint_prep.cu", ["-ffp-contract=off", *extra])]
    lib = link(d, objs, [HERE / "adjoint_host.cpp"], "libadjhost.so", extra)
    D = ctypes.POINTER(ctypes.c_double)
    lib.host_adjoint_backward.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, D, ctypes.c_int, D, D, D, D, D, D]
    lib.host_adjoint_backward.restype = ctypes.c_int
    return lib


@pytest.fixture(scope="module")
def host_adjoint(tmp_path_factory):
    return _build(tmp_path_factory.mktemp("adjhost"), contracted=False)


def _has_fma() -> bool:
    try:
        return " fma " in open("/proc/cpuinfo").read().replace("\n", " ")
    except OSError:
        return False


@pytest.fixture(scope="module")
def host_adjoint_contracted(tmp_path_factory):
    if not _has_fma():
        pytest.skip("the host has no fused multiply-add to model the device build with")
    return _build(tmp_path_factory.mktemp("adjhost_fma"), contracted=True)


BC = {"periodic": 0, "symmetric": 1}


def backward(lib, s, un, us, dts, seed):
    D = ctypes.POINTER(ctypes.c_double)

    def p(a):
        return None if a is None else a.ctypes.data_as(D)

    tab = None if s.eta_table is None else np.ascontiguousarray(s.eta_table, dtype=np.float64)
    gs = np.zeros_like(s.state)
    ge = np.zeros((s.nx, s.ny))
    un, us, dts, seed = (np.ascontiguousarray(x, dtype=np.float64) for x in (un, us, dts, seed))
    rc = lib.host_adjoint_backward(s.nx, s.ny, s.dx, s.dy, s.gamma, s.eps, s.eta, BC[s.bc],
                                   BC[s.bc_y] if s.bc_y else -1, p(tab), len(dts), p(un), p(us), p(dts), p(seed),
                                   p(gs), p(ge))
    assert rc == 0
    return gs, ge


def _dirs(setup, seed):
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(setup.state.shape)
    d[..., (1, 2, 3)] *= 1e-2
    d[..., (0, 4, 5, 6, 7)] *= 1e-3
    deta = rng.standard_normal((setup.nx, setup.ny)) * 1e-4
    return d, deta


def test_launch_rewrite_keeps_template_kernels_and_nested_arguments():
    src = ("  k1<<<dim3(f(n, 2), 2), T, 0, st>>>(a);\n"
           "  ytrans_kernel<BC_PERIODIC><<<g(x), 128, 0, st>>>(g, h(u, v));\n")
    out = rewrite_launches(src)
    assert out == ("  host_launch(dim3(f(n, 2), 2), T, [=]() { k1(a); });\n"
                   "  host_launch(g(x), 128, [=]() { ytrans_kernel<BC_PERIODIC>(g, h(u, v)); });\n")


@pytest.mark.parametrize("build", ["plain", "contracted"])
@pytest.mark.parametrize("with_table,shape,nsteps,bc,bc_y", [
    (False, (20, 18), 5, "periodic", None),
    (True, (26, 21), 6, "periodic", None),
    (False, (20, 18), 5, "symmetric", None),
    (True, (23, 26), 6, "symmetric", None),
    (True, (18, 21), 4, "periodic", "symmetric"),
    (False, (21, 17), 5, "symmetric", "periodic"),
])
def test_host_adjoint_matches_oracle_tangent(request, oracle, tangent, with_table, shape, nsteps, bc, bc_y, build):
    from resistivemhd_gpu_b200 import setups

    lib = request.getfixturevalue("host_adjoint" if build == "plain" else "host_adjoint_contracted")
    s = setups.random_smooth_state(*shape, seed=21, bc=bc, bc_y=bc_y, with_table=with_table)
    _, dts, crashed, un, us = oracle.run_keep_stages(s, s.state, nsteps)
    assert crashed == -1
    w = np.random.default_rng(5).standard_normal(s.state.shape)
    gs, ge = backward(lib, s, un, us, dts, w)
    ghost = np.ones(gs.shape[:2], bool)
    ghost[3:-3, 3:-3] = False
    mask = np.repeat(ghost[..., None], 8, axis=2)
    if bc == "symmetric":
        for c in (3, 4, s.nx - 6, s.nx - 5, s.nx - 4):
            mask[c, 2, 5] = False
    assert np.all(gs[mask] == 0)
    for k in range(3):
        d, deta = _dirs(s, 100 + k)
        _, dU = tangent.tangent(s, s.state, d, dts, deta=deta)
        jvp = float((w * dU).sum())
        vjp = float((gs * d).sum()) + float((ge * deta).sum())
        assert vjp == pytest.approx(jvp, rel=ADJ_REL, abs=1e-14)


def test_host_adjoint_unit_directions(host_adjoint, oracle, tangent):
    """Single components of dJ/dU_0 and dJ/d eta on a 12 x 12 interior with
    an eta table, against the tangent along unit directions."""
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(12, 12, seed=8, bc="periodic", with_table=True)
    _, dts, crashed, un, us = oracle.run_keep_stages(s, s.state, 3)
    assert crashed == -1
    w = np.random.default_rng(9).standard_normal(s.state.shape)
    gs, ge = backward(host_adjoint, s, un, us, dts, w)
    rng = np.random.default_rng(10)
    cells = [(i, j) for i in range(3, s.nx - 3) for j in range(3, s.ny - 3)]
    for t in rng.choice(len(cells), 6, replace=False):
        i, j = cells[t]
        for f in range(8):
            d = np.zeros_like(s.state)
            d[i, j, f] = 1.0
            _, dU = tangent.tangent(s, s.state, d, dts)
            assert gs[i, j, f] == pytest.approx(float((w * dU).sum()), rel=1e-9, abs=1e-12), (i, j, f)
        de = np.zeros((s.nx, s.ny))
        de[i, j] = 1.0
        _, dU = tangent.tangent(s, s.state, np.zeros_like(s.state), dts, deta=de)
        assert ge[i, j] == pytest.approx(float((w * dU).sum()), rel=1e-9, abs=1e-12), (i, j)


@pytest.mark.parametrize("build", ["plain", "contracted"])
def test_host_adjoint_on_the_harris_sheet(request, oracle, tangent, build):
    """Symmetric walls and the eta table of the Harris workload (64 x 32),
    where the fast and Alfven waves meet and the star states' N and D are
    differences of nearly equal terms.  The reverse recomputes them exactly
    rounded, as the forward does, so the gradient holds the tangent's 1e-10
    also when the rest of the reverse is contracted into fused multiply-adds
    as on the device (built that way, with N and D contracted too, this case
    was 6e-7 and 2e-6 off)."""
    from resistivemhd_gpu_b200 import setups

    lib = request.getfixturevalue("host_adjoint" if build == "plain" else "host_adjoint_contracted")
    s = setups.harris_sheet(64, 32)
    _, dts, crashed, un, us = oracle.run_keep_stages(s, s.state, 6)
    assert crashed == -1
    w = np.random.default_rng(3).standard_normal(s.state.shape)
    gs, ge = backward(lib, s, un, us, dts, w)
    for k in range(2):
        d, deta = _dirs(s, 200 + k)
        _, dU = tangent.tangent(s, s.state, d, dts, deta=deta)
        vjp = float((gs * d).sum() + (ge * deta).sum())
        assert vjp == pytest.approx(float((w * dU).sum()), rel=ADJ_REL, abs=1e-14)


def test_host_adjoint_against_central_differences(host_adjoint, oracle, tangent):
    """The misfit gradient of the host build against central differences
    (h = 1e-6 and 1e-7, the better one held to 1e-6) of the oracle's
    frozen-dt forward along localized directions of momentum and eta, as
    tests/test_gpu_adjoint.py checks the CUDA adjoint through the CUDA
    forward."""
    import copy

    from adjoint_harness import misfit_difference, misfit_seed
    from resistivemhd_gpu_b200 import setups

    s = setups.random_smooth_state(48, 48, seed=3, bc="periodic", with_table=True)
    eta0 = s.eta_table.copy()
    target = s.state.copy()
    final, dts, crashed, un, us = oracle.run_keep_stages(s, s.state, 10)
    assert crashed == -1
    gs, ge = backward(host_adjoint, s, un, us, dts, misfit_seed(final, target))

    def final_of(state, eta):
        s2 = copy.copy(s)
        s2.eta_table = eta
        return tangent.run_fixed_dt(s2, state, dts)

    rng = np.random.default_rng(7)
    for _ in range(4):
        d = np.zeros_like(s.state)
        de = np.zeros_like(eta0)
        i0, j0 = rng.integers(3, s.nx - 6), rng.integers(3, s.ny - 6)
        d[i0:i0 + 3, j0:j0 + 3, 1:3] = rng.standard_normal((3, 3, 2))
        de[i0:i0 + 3, j0:j0 + 3] = rng.standard_normal((3, 3)) * eta0[i0:i0 + 3, j0:j0 + 3]
        ad = float((gs * d).sum() + (ge * de).sum())
        errs = []
        for h in (1e-6, 1e-7):
            fd = misfit_difference(final_of(s.state + h * d, eta0 + h * de),
                                   final_of(s.state - h * d, eta0 - h * de), target) / (2 * h)
            errs.append(abs(fd - ad) / abs(ad))
        assert min(errs) <= 1e-6, (errs, ad)
