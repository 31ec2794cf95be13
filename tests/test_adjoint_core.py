"""CPU checks of the per-interface reverse-mode functions the CUDA adjoint
is built from (csrc/adjoint_core.cuh, compiled here for the host): the
HLLD flux reverse against the oracle's dual-number HLLD through the
dot-product identity <fb, J d> = <J^T fb, d>, and the primitive-recovery
reverse against central differences."""
import ctypes
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def core(tmp_path_factory):
    so = tmp_path_factory.mktemp("adjcore") / "libadjcore.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-o", str(so),
                    str(HERE / "adjoint_core_host.cpp")], check=True)
    lib = ctypes.CDLL(str(so))
    D = ctypes.POINTER(ctypes.c_double)
    lib.host_hlld_flux_adj.argtypes = [D, D, ctypes.c_double, ctypes.c_double, D, D, D]
    lib.host_basic_param.argtypes = [D, ctypes.c_double, ctypes.c_double, D]
    lib.host_basic_param_adj.argtypes = [D, ctypes.c_double, D, D]
    lib.host_muscl_states.argtypes = [D, D, D, D, ctypes.c_double, D, D]
    lib.host_muscl_states.restype = ctypes.c_uint
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _state(rng, u_shift=0.0, bx=None):
    # rho, u, v, w, bX, bY, bZ, p
    s = np.array([rng.uniform(0.5, 2.0), rng.normal() * 0.5 + u_shift, rng.normal() * 0.5, rng.normal() * 0.3,
                  rng.normal() * 0.7, rng.normal() * 0.7, rng.normal() * 0.4, rng.uniform(0.2, 2.0)])
    if bx is not None:
        s[4] = bx
    return s


@pytest.mark.parametrize("regime", ["subsonic", "supersonic_right", "supersonic_left", "zero_bn"])
def test_hlld_reverse_dot_product(core, tangent, regime):
    rng = np.random.default_rng(hash(regime) % 2**32)
    shift = {"subsonic": 0.0, "supersonic_right": 8.0, "supersonic_left": -8.0, "zero_bn": 0.0}[regime]
    gm, eps = 5.0 / 3.0, 1e-20
    worst = 0.0
    for _ in range(200):
        L = _state(rng, shift)
        R = _state(rng, shift)
        if regime == "zero_bn":
            L[4] = R[4] = 0.0
        else:
            R[4] = L[4]                         # one normal field per interface
        dL, dR = rng.standard_normal(8), rng.standard_normal(8)
        if regime == "zero_bn":
            dL[4] = dR[4] = 0.0
        fb = rng.standard_normal(8)
        _, df = tangent.hlld_jvp(L, R, dL, dR, gm, eps)
        Lb, Rb = np.zeros(8), np.zeros(8)
        core.host_hlld_flux_adj(_p(L), _p(R), gm, eps, _p(fb), _p(Lb), _p(Rb))
        lhs = float(fb @ df)
        rhs = float(Lb @ dL + Rb @ dR)
        scale = max(abs(lhs), np.abs(fb).max() * np.abs(df).max(), 1e-300)
        worst = max(worst, abs(lhs - rhs) / scale)
    assert worst < 1e-11, worst


def test_basic_param_reverse(core):
    rng = np.random.default_rng(4)
    gm = 5.0 / 3.0
    for _ in range(50):
        c = np.array([rng.uniform(0.5, 2), *rng.normal(size=6), 5.0 + rng.uniform()])
        qb = rng.standard_normal(8)
        cb = np.zeros(8)
        core.host_basic_param_adj(_p(c), gm, _p(qb), _p(cb))
        d = rng.standard_normal(8)
        h = 1e-6
        qp, qm = np.zeros(8), np.zeros(8)
        cp, cm = c + h * d, c - h * d
        core.host_basic_param(_p(cp), 0.3, gm, _p(qp))
        core.host_basic_param(_p(cm), 0.3, gm, _p(qm))
        fd = float(qb @ ((qp - qm) / (2 * h)))
        assert abs(fd - cb @ d) < 1e-7 * max(1.0, abs(fd))
