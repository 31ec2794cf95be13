"""The header-only C++ facade (include/rmhd2d.hpp) compiles against the C ABI
and, on a B200, a reference-style driver loop built on it reproduces the
oracle bit for bit and writes reference-format snapshots."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

DRIVER = r"""
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <vector>
#include "rmhd2d.hpp"

struct FromFile : rmhd2d::ResistiveMHD2D {
    std::vector<double> init;
    FromFile(const rmhd2d_config &c, std::vector<double> u) : rmhd2d::ResistiveMHD2D(c), init(std::move(u)) {}
    void initializeU() override { hostU() = init; }
};

int main(int argc, char **argv) {
    // argv: in.bin outdir nx ny dx dy eta steps
    int nx = std::atoi(argv[3]), ny = std::atoi(argv[4]);
    rmhd2d_config cfg; rmhd2d_config_default(&cfg);
    cfg.nx = nx; cfg.ny = ny; cfg.dx = std::atof(argv[5]); cfg.dy = std::atof(argv[6]);
    cfg.eta = std::atof(argv[7]);
    int steps = std::atoi(argv[8]);
    std::vector<double> u((size_t)nx * ny * 8);
    std::ifstream f(argv[1], std::ios::binary);
    f.read(reinterpret_cast<char *>(u.data()), u.size() * sizeof(double));
    try {
        FromFile run(cfg, u);
        run.initialize();
        double totalTime = 0.0;
        for (int step = 0; step < steps; ++step) {
            run.oneStepRK2();
            if (run.checkCalculationIsCrashed()) { std::printf("crashed %d\n", step); return 1; }
            totalTime += run.dt();
        }
        run.save(argv[2], "ot", steps);
        std::printf("%.17g\n", totalTime);
    } catch (const rmhd2d::Error &e) {
        std::printf("error %d %s\n", e.status, e.what());
        return 10 + e.status;
    }
    return 0;
}
"""


def build_driver(tmp_path: Path) -> Path:
    from resistivemhd_gpu_b200 import _lib

    _lib.load()  # library present
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    libdir = ROOT / "resistivemhd_gpu_b200"
    subprocess.run(["g++", "-std=c++17", "-O1", str(src), "-I", str(ROOT / "include"), "-L", str(libdir),
                    "-lrmhd2d", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True, capture_output=True)
    return exe


def test_facade_compiles_and_reports_missing_device(tmp_path):
    import torch

    exe = build_driver(tmp_path)
    if torch.cuda.is_available():
        pytest.skip("a GPU is present; covered by the gpu test")
    from resistivemhd_gpu_b200 import setups

    s = setups.orszag_tang(8)
    s.state.tofile(tmp_path / "in.bin")
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path), str(s.nx), str(s.ny), repr(s.dx),
                        repr(s.dy), repr(s.eta), "2"], capture_output=True, text=True)
    assert r.returncode == 13, r.stdout + r.stderr   # 10 + RMHD2D_ERR_NO_DEVICE
    assert "no" in r.stdout


@pytest.mark.gpu
def test_facade_driver_matches_oracle(gpu, oracle, tmp_path):
    from resistivemhd_gpu_b200 import read_snapshot, setups

    exe = build_driver(tmp_path)
    s = setups.orszag_tang(48)
    s.state.tofile(tmp_path / "in.bin")
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path), str(s.nx), str(s.ny), repr(s.dx),
                        repr(s.dy), repr(s.eta), "6"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    ref, dts, _ = oracle.run(s, s.state, 6)
    out = read_snapshot(str(tmp_path / "ot_6.bin"), s.nx, s.ny)
    assert np.array_equal(out, ref)
    assert float(r.stdout.strip()) == pytest.approx(dts.sum(), rel=1e-15)
