"""The reference drivers' main loop (snapshots every recordStep steps and the
"step,totalTime" log) in Python (resistivemhd_gpu_b200.driver) and in the C++
facade (rmhd2d::runLikeReference): snapshots are the oracle's states in the
save() format, the log has the reference's format, and a crashed state stops
the loop as the reference's does."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

CXX_DRIVER = r"""
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>
#include "rmhd2d.hpp"

struct FromFile : rmhd2d::ResistiveMHD2D {
    std::vector<double> init;
    FromFile(const rmhd2d_config &c, std::vector<double> u) : rmhd2d::ResistiveMHD2D(c), init(std::move(u)) {}
    void initializeU() override { hostU() = init; }
};

int main(int argc, char **argv) {
    // argv: in.bin outdir nx ny dx dy eta totalStep recordStep
    int nx = std::atoi(argv[3]), ny = std::atoi(argv[4]);
    rmhd2d_config cfg; rmhd2d_config_default(&cfg);
    cfg.nx = nx; cfg.ny = ny; cfg.dx = std::atof(argv[5]); cfg.dy = std::atof(argv[6]);
    cfg.eta = std::atof(argv[7]);
    std::vector<double> u((size_t)nx * ny * 8);
    std::ifstream f(argv[1], std::ios::binary);
    f.read(reinterpret_cast<char *>(u.data()), u.size() * sizeof(double));
    FromFile run(cfg, u);
    run.initialize();
    std::ofstream logfile(std::string(argv[2]) + "/log_cxx.txt");
    double totalTime = 0.0;
    int stopped = rmhd2d::runLikeReference(run, std::atoi(argv[8]), std::atoi(argv[9]), argv[2], "cxx", logfile,
                                           totalTime, false);
    std::cout << stopped << "\n";
    return 0;
}
"""


def _compile(tmp_path):
    exe = tmp_path / "driver_cxx"
    lib = ROOT / "resistivemhd_gpu_b200"
    subprocess.run(["g++", "-std=c++17", "-O1", "-x", "c++", "-", "-I", str(ROOT / "include"), "-L", str(lib),
                    "-lrmhd2d", f"-Wl,-rpath,{lib}", "-o", str(exe)], input=CXX_DRIVER.encode(), check=True)
    return exe


def test_cxx_driver_loop_compiles(tmp_path):
    from resistivemhd_gpu_b200 import build

    build.build()
    assert _compile(tmp_path).exists()


@pytest.mark.gpu
def test_driver_loop_snapshots_log_and_crash_stop(gpu, oracle, tmp_path):
    from resistivemhd_gpu_b200 import Solver, driver, read_snapshot, setups

    s = setups.orszag_tang(48)
    with Solver.from_setup(s, precision="fp64_exact") as sol:
        res = driver.run_like_reference(sol, 12, 4, str(tmp_path / "py"), "ot", echo=False)
    assert res["stopped_at"] == 13 and not res["crashed"]
    _, dts, _ = oracle.run(s, s.state, 12)
    lines = (tmp_path / "py" / "log_ot.txt").read_text().splitlines()
    want_t = [0.0, dts[:4].sum(), dts[:8].sum(), dts[:12].sum()]
    assert lines == [f"{k},{'%.4g' % t}" for k, t in zip((0, 4, 8, 12), want_t)]
    for k in (0, 4, 8, 12):
        ref = oracle.run(s, s.state, k)[0] if k else oracle.boundary(s, s.state)
        got = read_snapshot(str(tmp_path / "py" / f"ot_{k}.bin"), s.nx, s.ny)
        assert np.array_equal(got, ref)
    # the loop steps once more after the last record (steps 0 .. 12 each take a step)
    _, dts13, _ = oracle.run(s, s.state, 13)
    assert res["total_time"] == pytest.approx(dts13.sum(), rel=1e-15)

    # a NaN energy stops the loop after the step that reads it
    bad = s.state.copy()
    bad[10, 10, 7] = np.nan
    s2 = setups.Setup(s.name, bad, s.dx, s.dy, s.gamma, s.cfl, s.eps, s.eta, None, s.bc)
    with Solver.from_setup(s2, precision="fp64_exact") as sol:
        res = driver.run_like_reference(sol, 12, 4, str(tmp_path / "bad"), "ot", echo=False)
    assert res["crashed"] and res["stopped_at"] == 0
    assert (tmp_path / "bad" / "log_ot.txt").read_text().splitlines() == ["0,0"]

    # the C++ facade's loop writes the same log and snapshots
    exe = _compile(tmp_path)
    inp = tmp_path / "in.bin"
    np.ascontiguousarray(s.state).tofile(inp)
    out = tmp_path / "cxx"
    out.mkdir()
    r = subprocess.run([str(exe), str(inp), str(out), str(s.nx), str(s.ny), repr(s.dx), repr(s.dy), repr(s.eta),
                        "12", "4"], capture_output=True, text=True, check=True)
    assert r.stdout.strip() == "13"
    assert (out / "log_cxx.txt").read_text().splitlines() == lines
    for k in (0, 4, 8, 12):
        assert (out / f"cxx_{k}.bin").read_bytes() == (tmp_path / "py" / f"ot_{k}.bin").read_bytes()
