"""The step/time log of the reference drivers' main loop
(examples2D/plasmoid/main_plasmoid.cu:297-329 writes "step,totalTime" with
std::setprecision(4)): the Python driver's formatting equals the C++
stream's for the same doubles, so logs written by
resistivemhd_gpu_b200.driver.run_like_reference and by
rmhd2d::runLikeReference (include/rmhd2d.hpp) read the same as the
reference's."""
import subprocess

import numpy as np

PROGRAM = r"""
#include <cstdio>
#include <iomanip>
#include <iostream>
#include <string>
int main() {
    double x;
    while (std::scanf("%lf", &x) == 1) std::cout << std::setprecision(4) << x << "\n";
    return 0;
}
"""


def _values():
    rng = np.random.default_rng(11)
    fixed = [0.0, 1.0, 0.1, 0.5, 2.0, 10.0, 123.456, 1234.5, 12345.0, 99999.0, 1e-5, 1.23456e-7, 3.14159265358979,
             2.5e10, 0.00012345, 0.001, 9.9995, 9.99949, 1e100, 5e-324]
    rand = [float(v) for v in 10.0 ** rng.uniform(-8, 8, 200) * rng.choice([1.0, 1.0 + 1e-9], 200)]
    return fixed + rand


def test_python_log_format_equals_cxx_setprecision4(tmp_path):
    from resistivemhd_gpu_b200.driver import _fmt4

    src = tmp_path / "fmt.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "fmt"
    subprocess.run(["g++", "-std=c++17", str(src), "-o", str(exe)], check=True, capture_output=True)
    vals = _values()
    stdin = "\n".join(repr(v) for v in vals) + "\n"
    out = subprocess.run([str(exe)], input=stdin, check=True, capture_output=True, text=True).stdout.split()
    assert len(out) == len(vals)
    for v, cxx in zip(vals, out):
        assert _fmt4(v) == cxx, (v, _fmt4(v), cxx)
