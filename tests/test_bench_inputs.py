"""CPU checks of what bench.py reads besides the GPU: the committed profile
summaries it takes the DRAM traffic and the flop count from, its misfit
difference, the control-block size its e2e byte count uses, and the
synthetic set-ups every benchmark and parity run starts from
(divergence-free to round-off, positive density and pressure)."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


@pytest.mark.parametrize("precision", ["fp64_fast", "fp64_exact", "fp32_bulk"])
def test_profile_traffic_is_readable(precision):
    import bench

    t = bench.traffic_from_profile(f"harris_2048x1024_{precision}")
    assert t is not None and set(t) == {"stage1", "stage2"}
    alg = bench.algorithmic_bytes(bench.workload("harris")[0])
    for k in ("stage1", "stage2"):
        # DRAM traffic of a launch within a few tens of percent of its algorithmic bytes
        assert 0.5 * alg[k] < t[k] < 1.5 * alg[k], (k, t[k], alg[k])


def test_profile_flop_count_is_readable():
    import bench

    f = bench.flops_from_profile("harris_2048x1024")
    assert f is not None and 2000 < f < 6000


def test_misfit_difference_is_the_difference_of_misfits():
    import bench

    rng = np.random.default_rng(0)
    shape = (20, 18, 8)
    t, a, b = rng.standard_normal(shape), rng.standard_normal(shape), rng.standard_normal(shape)
    fields = [0, 4, 5, 6]

    def J(x):
        d = x[3:-3, 3:-3, fields] - t[3:-3, 3:-3, fields]
        return 0.5 * float((d * d).sum())

    assert bench._misfit_difference(a, b, t, fields) == pytest.approx(J(a) - J(b), rel=1e-12)


def _div_b(state, dx, dy):
    return (state[3:-3, 3:-3, 4] - state[2:-4, 3:-3, 4]) / dx + (state[3:-3, 3:-3, 5] - state[3:-3, 2:-4, 5]) / dy


def _pressure(s):
    u = s.state
    bxc = 0.5 * (u[1:, :, 4] + u[:-1, :, 4])[2:-3, 3:-3]
    byc = 0.5 * (u[:, 1:, 5] + u[:, :-1, 5])[3:-3, 2:-3]
    c = u[3:-3, 3:-3]
    ke = 0.5 * (c[..., 1] ** 2 + c[..., 2] ** 2 + c[..., 3] ** 2) / c[..., 0]
    return (s.gamma - 1.0) * (c[..., 7] - ke - 0.5 * (bxc ** 2 + byc ** 2 + c[..., 6] ** 2))


@pytest.mark.parametrize("make", [
    lambda st: st.orszag_tang(64),
    lambda st: st.harris_sheet(128, 64),
    lambda st: st.plasmoid_sheet(256, 128),
    lambda st: st.kelvin_helmholtz(64),
    lambda st: st.ot_adjoint(64),
    lambda st: st.random_smooth_state(30, 26, seed=3, bc="symmetric", with_table=True),
])
def test_setups_are_divergence_free_and_positive(make):
    from resistivemhd_gpu_b200 import setups

    s = make(setups)
    assert np.isfinite(s.state).all()
    scale = np.abs(s.state[..., 4:6]).max() / min(s.dx, s.dy)
    assert np.abs(_div_b(s.state, s.dx, s.dy)).max() <= 1e-12 * max(scale, 1.0)
    assert s.state[3:-3, 3:-3, 0].min() > 0
    assert _pressure(s).min() > 0
    if s.eta_table is not None:
        assert s.eta_table.min() >= 0 and s.eta >= s.eta_table.max()


def test_control_block_size_matches_the_library(tmp_path):
    """The e2e line counts the control block each synchronising query reads
    back; that count is sizeof(rmhd2d::Control) of the library's own header."""
    import subprocess

    import bench

    src = tmp_path / "size.cpp"
    src.write_text('#include <cstdio>\n#include "rmhd2d_internal.h"\n'
                   'int main() { std::printf("%zu\\n", sizeof(rmhd2d::Control)); return 0; }\n')
    exe = tmp_path / "size"
    subprocess.run(["g++", "-std=c++17", str(src), "-I", str(ROOT / "resistivemhd_gpu_b200" / "csrc"), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert int(out) == bench.CONTROL_BLOCK_BYTES
