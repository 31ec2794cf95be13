"""Python access to the parity oracles.  TEST INFRASTRUCTURE ONLY.

* ``OracleLib`` -- ctypes binding of the C restatement ``rmhd2d_oracle.c``
  (built into ``oracle/liborc.so`` by ``build()``).
* ``run_reference`` -- runs the reference's own step built by
  ``oracle/build_ref.py`` (``oracle/_ref/ref_{cpu,gpu}_{periodic,symmetric}``)
  on a state and returns the final state, the per-step dt and the timing.
* ``run_mc_boundary`` / ``run_mc_ct`` -- run the multi-GPU library's own wall
  functions and CT-Contact closing CT (``oracle/_ref/mc_host``) on given
  inputs.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference legs may import this module.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liborc.so"
TANGENT_LIB = HERE / "libtangent.so"
REF_DIR = HERE / "_ref"

BC = {"periodic": 0, "symmetric": 1, "zero_gradient": 2, "wall": 3, "flare": 4}


class _Params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("gamma", ctypes.c_double), ("cfl", ctypes.c_double), ("eps", ctypes.c_double),
        ("eta", ctypes.c_double), ("eta_table", ctypes.POINTER(ctypes.c_double)),
        ("bc", ctypes.c_int), ("bc_y", ctypes.c_int), ("ct_contact", ctypes.c_int),
    ]


def build(verbose: bool = False) -> Path:
    """Compile the C restatement (no FMA contraction) into oracle/liborc.so."""
    src = HERE / "rmhd2d_oracle.c"
    if LIB.exists() and LIB.stat().st_mtime >= max(src.stat().st_mtime, (HERE / "rmhd2d_oracle.h").stat().st_mtime):
        return LIB
    cmd = ["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-Wall", "-o", str(LIB), str(src), "-lm"]
    subprocess.run(cmd, check=True, capture_output=not verbose)
    return LIB


def build_tangent(verbose: bool = False) -> Path:
    """Compile the templated restatement (rmhd2d_tangent.cpp) into
    oracle/libtangent.so."""
    src = HERE / "rmhd2d_tangent.cpp"
    deps = [src, HERE / "rmhd2d_oracle.h"]
    if TANGENT_LIB.exists() and TANGENT_LIB.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return TANGENT_LIB
    cmd = ["g++", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           "-Wall", "-o", str(TANGENT_LIB), str(src), "-lm"]
    subprocess.run(cmd, check=True, capture_output=not verbose)
    return TANGENT_LIB


class TangentLib:
    """The oracle step as a template, on doubles with given dts and on dual
    numbers: the exact directional derivative of the frozen-dt map, against
    which the CUDA adjoint is checked."""

    def __init__(self):
        build_tangent()
        self.lib = ctypes.CDLL(str(TANGENT_LIB))
        P = ctypes.POINTER(_Params)
        D = ctypes.POINTER(ctypes.c_double)
        self.lib.orc_run_fixed_dt.argtypes = [P, D, ctypes.c_int, D, ctypes.c_int]
        self.lib.orc_tangent_run.argtypes = [P, D, D, D, ctypes.c_int, D]
        self.lib.orc_hlld_jvp.argtypes = [D, D, D, D, ctypes.c_double, ctypes.c_double, D, D]
        self.lib.orc_count_ops.argtypes = [P, D, ctypes.c_int, D, ctypes.c_int, ctypes.POINTER(ctypes.c_ulonglong)]

    @staticmethod
    def _d(a):
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def run_fixed_dt(self, setup, state, dts, apply_boundary=True):
        keep = []
        p = OracleLib._params(setup, keep)
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        d = np.ascontiguousarray(dts, dtype=np.float64)
        self.lib.orc_run_fixed_dt(ctypes.byref(p), self._d(s), len(d), self._d(d), int(bool(apply_boundary)))
        return s

    def tangent(self, setup, state, dstate, dts, deta=None):
        """(U_N, dU_N) for the run from `state` (before its boundary) with the
        given dts, along the direction (dstate, deta)."""
        keep = []
        p = OracleLib._params(setup, keep)
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        ds = np.ascontiguousarray(dstate, dtype=np.float64).copy()
        d = np.ascontiguousarray(dts, dtype=np.float64)
        de = None if deta is None else np.ascontiguousarray(deta, dtype=np.float64)
        self.lib.orc_tangent_run(ctypes.byref(p), self._d(s), self._d(ds), None if de is None else self._d(de),
                                 len(d), self._d(d))
        return s, ds

    def count_ops(self, setup, state, dts, apply_boundary=True):
        """(U_N, counts) of the run on the operation-counting scalar; counts
        maps add (incl. sub), mul, div, sqrt, abs, cmp to totals over the
        whole array and all steps."""
        keep = []
        p = OracleLib._params(setup, keep)
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        d = np.ascontiguousarray(dts, dtype=np.float64)
        c = (ctypes.c_ulonglong * 6)()
        self.lib.orc_count_ops(ctypes.byref(p), self._d(s), len(d), self._d(d), int(bool(apply_boundary)), c)
        return s, dict(zip(("add", "mul", "div", "sqrt", "abs", "cmp"), (int(v) for v in c)))

    def hlld_jvp(self, L, R, dL, dR, gamma, eps):
        f, df = np.zeros(8), np.zeros(8)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (L, R, dL, dR)]
        self.lib.orc_hlld_jvp(*[self._d(a) for a in arrs], gamma, eps, self._d(f), self._d(df))
        return f, df


class OracleLib:
    def __init__(self):
        build()
        self.lib = ctypes.CDLL(str(LIB))
        P = ctypes.POINTER(_Params)
        D = ctypes.POINTER(ctypes.c_double)
        self.lib.orc_calc_dt.argtypes = [P, D]
        self.lib.orc_calc_dt.restype = ctypes.c_double
        self.lib.orc_is_crashed.argtypes = [P, D]
        self.lib.orc_boundary.argtypes = [P, D]
        self.lib.orc_run.argtypes = [P, D, ctypes.c_int, D]
        self.lib.orc_run.restype = ctypes.c_int
        self.lib.orc_run_keep_stages.argtypes = [P, D, ctypes.c_int, D, D, D]
        self.lib.orc_run_keep_stages.restype = ctypes.c_int
        self.lib.orc_contact_ct_work_doubles.argtypes = [ctypes.c_int, ctypes.c_int]
        self.lib.orc_contact_ct_work_doubles.restype = ctypes.c_size_t
        self.lib.orc_contact_ct.argtypes = [P, D, D, D, D, D, D, D, ctypes.c_double, D, D]

    @staticmethod
    def _params(setup, eta_keep):
        tab = None
        if setup.eta_table is not None:
            tab = np.ascontiguousarray(setup.eta_table, dtype=np.float64)
            eta_keep.append(tab)
        p = _Params(setup.nx, setup.ny, setup.dx, setup.dy, setup.gamma, setup.cfl, setup.eps,
                    setup.eta, tab.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if tab is not None else None,
                    BC[setup.bc], BC[getattr(setup, "bc_y", None) or setup.bc],
                    1 if getattr(setup, "ct", "stage1") == "contact" else 0)
        return p

    def boundary(self, setup, state: np.ndarray) -> np.ndarray:
        keep = []
        p = self._params(setup, keep)
        out = np.ascontiguousarray(state, dtype=np.float64).copy()
        self.lib.orc_boundary(ctypes.byref(p), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def contact_ct(self, setup, u_old, f_old, g_old, u_now, f_now, g_now, bx_old, by_old, dt: float) -> np.ndarray:
        """The closing CT of the CT-Contact step on given inputs
        (orc_contact_ct): returns u_now with its face B replaced."""
        keep = []
        p = self._params(setup, keep)
        D = ctypes.POINTER(ctypes.c_double)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u_old, f_old, g_old, f_now, g_now, bx_old,
                                                                    by_old)]
        out = np.ascontiguousarray(u_now, dtype=np.float64).copy()
        work = np.empty(self.lib.orc_contact_ct_work_doubles(setup.nx, setup.ny), dtype=np.float64)
        self.lib.orc_contact_ct(ctypes.byref(p), *[a.ctypes.data_as(D) for a in arrs], float(dt),
                                out.ctypes.data_as(D), work.ctypes.data_as(D))
        return out

    def calc_dt(self, setup, state: np.ndarray) -> float:
        keep = []
        p = self._params(setup, keep)
        s = np.ascontiguousarray(state, dtype=np.float64)
        return self.lib.orc_calc_dt(ctypes.byref(p), s.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def run(self, setup, state: np.ndarray, nsteps: int, apply_boundary: bool = True):
        """Returns (final_state, dts, crashed_at) after nsteps RK2 steps."""
        keep = []
        p = self._params(setup, keep)
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        dp = s.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if apply_boundary:
            self.lib.orc_boundary(ctypes.byref(p), dp)
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        rc = self.lib.orc_run(ctypes.byref(p), dp, nsteps, dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc < 0:
            raise MemoryError("oracle work allocation failed")
        crashed_at = rc - 1 if rc > 0 else -1
        return s, dts[:nsteps], crashed_at


    def run_keep_stages(self, setup, state: np.ndarray, nsteps: int, apply_boundary: bool = True):
        """As run, plus the trajectory a discrete adjoint reverses: (final_state,
        dts, crashed_at, Un, Ustar), Un[s] the state step s starts from and
        Ustar[s] its stage-1 state after the boundary pass."""
        keep = []
        p = self._params(setup, keep)
        s = np.ascontiguousarray(state, dtype=np.float64).copy()
        D = ctypes.POINTER(ctypes.c_double)
        dp = s.ctypes.data_as(D)
        if apply_boundary:
            self.lib.orc_boundary(ctypes.byref(p), dp)
        n = max(nsteps, 1)
        dts = np.zeros(n, dtype=np.float64)
        un = np.zeros((n,) + s.shape, dtype=np.float64)
        us = np.zeros((n,) + s.shape, dtype=np.float64)
        rc = self.lib.orc_run_keep_stages(ctypes.byref(p), dp, nsteps, dts.ctypes.data_as(D), un.ctypes.data_as(D),
                                          us.ctypes.data_as(D))
        if rc < 0:
            raise MemoryError("oracle work allocation failed")
        crashed_at = rc - 1 if rc > 0 else -1
        return s, dts[:nsteps], crashed_at, un[:nsteps], us[:nsteps]


def reference_binary(kind: str, bc: str) -> Path:
    return REF_DIR / f"ref_{kind}_{bc}"


MC_BINARY = REF_DIR / "mc_host"
# wall pairs of the multi-GPU library's step variants, as (x wall, y wall) of
# this project's configuration; the library's symmetricBoundaryY2nd is the
# zero-gradient copy
MC_PAIRS = {"periodic_periodic": ("periodic", "periodic"), "periodic_wall": ("periodic", "wall"),
            "periodic_zerogradient": ("periodic", "zero_gradient"), "flare_wall": ("flare", "wall")}


def _mc_env(setup, dt: float = 0.0) -> dict:
    env = dict(os.environ)
    env.update({"REF_NX": str(setup.nx), "REF_NY": str(setup.ny), "REF_DX": repr(setup.dx),
                "REF_DY": repr(setup.dy), "REF_GAMMA": repr(setup.gamma), "REF_EPS": repr(setup.eps),
                "REF_ETA": repr(setup.eta), "MC_DT": repr(float(dt)), "OMP_NUM_THREADS": "1"})
    return env


def run_mc_boundary(setup, state: np.ndarray, pair: str) -> np.ndarray:
    """The multi-GPU library's own ghost fill for a wall pair (sendrecv_U on
    one rank, then its x and y wall functions), built by build_ref.build_mc."""
    if not MC_BINARY.exists():
        raise FileNotFoundError(f"{MC_BINARY} not built (oracle/build_ref.py mc)")
    with tempfile.TemporaryDirectory(dir=os.environ.get("RMHD_TMPDIR")) as td:
        td = Path(td)
        np.ascontiguousarray(state, dtype=np.float64).tofile(td / "in.bin")
        r = subprocess.run([str(MC_BINARY), "boundary", pair, str(td / "in.bin"), str(td / "out.bin")],
                           env=_mc_env(setup), capture_output=True, text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(f"mc_host boundary failed ({r.returncode}): {r.stderr[-2000:]}")
        return np.fromfile(td / "out.bin", dtype=np.float64).reshape(state.shape)


def run_mc_ct(setup, u_old, f_old, g_old, u_now, f_now, g_now, bx_old, by_old, dt: float) -> np.ndarray:
    """The multi-GPU library's own CT-Contact closing CT (CT::setOldFlux2D,
    CT::setNowFlux2D, CT::divBClean) on given inputs; returns u_now with the
    face B it writes."""
    if not MC_BINARY.exists():
        raise FileNotFoundError(f"{MC_BINARY} not built (oracle/build_ref.py mc)")
    with tempfile.TemporaryDirectory(dir=os.environ.get("RMHD_TMPDIR")) as td:
        td = Path(td)
        for name, a in (("u_old", u_old), ("f_old", f_old), ("g_old", g_old), ("u_now", u_now), ("f_now", f_now),
                        ("g_now", g_now), ("bx_old", bx_old), ("by_old", by_old)):
            np.ascontiguousarray(a, dtype=np.float64).tofile(td / name)
        env = _mc_env(setup, dt)
        if setup.eta_table is not None:
            np.ascontiguousarray(setup.eta_table, dtype=np.float64).tofile(td / "eta.bin")
            env["REF_ETA_TABLE"] = str(td / "eta.bin")
        r = subprocess.run([str(MC_BINARY), "ct", str(td), str(td / "out.bin")], env=env, capture_output=True,
                           text=True, timeout=600)
        if r.returncode != 0:
            raise RuntimeError(f"mc_host ct failed ({r.returncode}): {r.stderr[-2000:]}")
        return np.fromfile(td / "out.bin", dtype=np.float64).reshape(np.shape(u_now))


def run_reference(setup, state: np.ndarray, n_timed: int, n_warmup: int = 0, kind: str = "cpu",
                  threads: int | None = None, timeout: float = 1800.0):
    """Run the reference's own step (built by build_ref.py) from ``state``
    (boundary applied inside, as the reference's initializeU does).
    Returns (final_state, dts, info_dict)."""
    exe = reference_binary(kind, setup.bc)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} not built (oracle/build_ref.py)")
    env = dict(os.environ)
    env.update({
        "REF_NX": str(setup.nx), "REF_NY": str(setup.ny), "REF_DX": repr(setup.dx), "REF_DY": repr(setup.dy),
        "REF_GAMMA": repr(setup.gamma), "REF_CFL": repr(setup.cfl), "REF_EPS": repr(setup.eps),
        "REF_ETA": repr(setup.eta),
    })
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory(dir=os.environ.get("RMHD_TMPDIR")) as td:
        td = Path(td)
        np.ascontiguousarray(state, dtype=np.float64).tofile(td / "in.bin")
        if setup.eta_table is not None:
            np.ascontiguousarray(setup.eta_table, dtype=np.float64).tofile(td / "eta.bin")
            env["REF_ETA_TABLE"] = str(td / "eta.bin")
        else:
            env["REF_ETA_TABLE"] = ""
        r = subprocess.run([str(exe), str(td / "in.bin"), str(td / "out.bin"), str(n_warmup), str(n_timed),
                            str(td / "dts.bin")], env=env, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"{exe.name} failed ({r.returncode}): {r.stderr[-2000:]}")
        info = json.loads(r.stdout.strip().splitlines()[-1])
        out = np.fromfile(td / "out.bin", dtype=np.float64).reshape(setup.nx, setup.ny, 8)
        dts = np.fromfile(td / "dts.bin", dtype=np.float64)
    return out, dts, info
