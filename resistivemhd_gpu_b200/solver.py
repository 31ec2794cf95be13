"""Python host interface of the B200 resistive-MHD step.

``Solver`` wraps one ``rmhd2d_solver`` of the C ABI.  ``ResistiveMHD2D``
mirrors the reference's class of the same name
(ResistiveMHD_singleGPU_thrust/lib_ResistiveMHD_2D_GPU_periodicXY/
resistiveMHD_2D.hpp:9-52): ``initializeU`` (overridden by the user, as the
reference's drivers do), ``oneStepRK2``, ``calculateDt``, ``save``, ``getU``
and ``checkCalculationIsCrashed``, plus the reference's globals ``dt`` and
``totalTime`` as attributes.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

_DP = ctypes.POINTER(ctypes.c_double)


def _as_f64(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Solver:
    """One solver instance on one CUDA device.

    ``nx``, ``ny`` include 3 ghost layers per side.  ``bc`` names the x walls
    and, unless ``bc_y`` is given, the y walls too: "periodic", "symmetric",
    "zero_gradient", "flare" (x only) or "wall" (y only).  ``precision`` is
    "fp64_exact" (bit-for-bit the reference's IEEE binary64 arithmetic),
    "fp64_fast" (FMA contraction) or "fp32_bulk" (FP32 reconstruction and
    fan, FP64 stresses, update and dt).  ``ct`` is "stage1" (the single-GPU
    library's stage-1 EMF) or "contact" (CT-Contact).  ``stream`` may be a
    CUDA stream handle (int) to enqueue on."""

    def __init__(self, nx: int, ny: int, dx: float, dy: float, *, gamma: float = 5.0 / 3.0, cfl: float = 0.4,
                 eps: float = 1e-20, eta: float = 0.0, bc: str = "periodic", bc_y: str | None = None,
                 precision: str = "fp64_exact", device: int = 0, stream: int | None = None, ct: str = "stage1"):
        lib = _lib.load()
        cfg = _lib.Config()
        lib.rmhd2d_config_default(ctypes.byref(cfg))
        cfg.nx, cfg.ny, cfg.dx, cfg.dy = int(nx), int(ny), float(dx), float(dy)
        cfg.gamma_mhd, cfg.cfl, cfg.eps, cfg.eta = float(gamma), float(cfl), float(eps), float(eta)
        if bc not in _lib.BC or (bc_y is not None and bc_y not in _lib.BC):
            raise ValueError(f"unknown boundary kind {bc!r} / {bc_y!r}")
        if precision not in _lib.PRECISION:
            raise ValueError(f"unknown precision {precision!r}")
        cfg.bc = _lib.BC[bc]
        cfg.bc_y = -1 if bc_y is None else _lib.BC[bc_y]
        cfg.precision = _lib.PRECISION[precision]
        cfg.device = int(device)
        cfg.stream = stream
        if ct not in _lib.CT:
            raise ValueError(f"unknown CT scheme {ct!r}")
        cfg.ct_scheme = _lib.CT[ct]
        h = ctypes.c_void_p()
        _lib.check(lib.rmhd2d_create(ctypes.byref(cfg), ctypes.byref(h)), None)
        self._lib = lib
        self._h = h
        self._owned = True
        self.nx, self.ny = int(nx), int(ny)
        self.bc, self.bc_y, self.precision = bc, (bc if bc_y is None else bc_y), precision

    @staticmethod
    def make_config(nx, ny, dx, dy, *, gamma=5.0 / 3.0, cfl=0.4, eps=1e-20, eta=0.0, bc="periodic", bc_y=None,
                    precision="fp64_exact", device=0, ct="stage1") -> "_lib.Config":
        lib = _lib.load()
        cfg = _lib.Config()
        lib.rmhd2d_config_default(ctypes.byref(cfg))
        cfg.nx, cfg.ny, cfg.dx, cfg.dy = int(nx), int(ny), float(dx), float(dy)
        cfg.gamma_mhd, cfg.cfl, cfg.eps, cfg.eta = float(gamma), float(cfl), float(eps), float(eta)
        cfg.bc = _lib.BC[bc]
        cfg.bc_y = -1 if bc_y is None else _lib.BC[bc_y]
        cfg.precision = _lib.PRECISION[precision]
        cfg.device = int(device)
        cfg.ct_scheme = _lib.CT[ct]
        return cfg

    @classmethod
    def _member(cls, handle: ctypes.c_void_p, nx: int, ny: int) -> "Solver":
        """Non-owning view of a batch member."""
        s = cls.__new__(cls)
        s._lib = _lib.load()
        s._h = handle
        s._owned = False
        s.nx, s.ny = int(nx), int(ny)
        return s

    @classmethod
    def from_setup(cls, setup, precision: str = "fp64_exact", device: int = 0, apply_boundary: bool = True,
                   stream: int | None = None) -> "Solver":
        s = cls(setup.nx, setup.ny, setup.dx, setup.dy, gamma=setup.gamma, cfl=setup.cfl, eps=setup.eps,
                eta=setup.eta, bc=setup.bc, bc_y=setup.bc_y, precision=precision, device=device, stream=stream,
                ct=getattr(setup, "ct", "stage1"))
        if setup.eta_table is not None:
            s.set_eta_table(setup.eta_table)
        s.set_state(setup.state, apply_boundary=apply_boundary)
        return s

    # -- lifetime --
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            if getattr(self, "_owned", True):
                self._lib.rmhd2d_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, st: int) -> None:
        _lib.check(st, self._h)

    # -- state --
    def set_state(self, state: np.ndarray, apply_boundary: bool = True) -> None:
        a = _as_f64(state)
        if a.size != self.nx * self.ny * 8:
            raise ValueError(f"state must hold {self.nx}x{self.ny}x8 doubles, got shape {a.shape}")
        self._ck(self._lib.rmhd2d_set_state(self._h, a.ctypes.data_as(_DP), int(bool(apply_boundary))))

    def set_state_device(self, device_ptr: int, apply_boundary: bool = True) -> None:
        self._ck(self._lib.rmhd2d_set_state_device(self._h, ctypes.c_void_p(device_ptr), int(bool(apply_boundary))))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.nx, self.ny, 8), dtype=np.float64)
        if not (out.flags.c_contiguous and out.dtype == np.float64 and out.size == self.nx * self.ny * 8):
            raise ValueError("out must be a C-contiguous float64 array of nx*ny*8 elements")
        self._ck(self._lib.rmhd2d_get_state(self._h, out.ctypes.data_as(_DP)))
        return out

    def set_eta_table(self, eta: np.ndarray | None) -> None:
        if eta is None:
            self._ck(self._lib.rmhd2d_set_eta_table(self._h, None))
            return
        a = _as_f64(eta)
        if a.size != self.nx * self.ny:
            raise ValueError("eta table must hold nx*ny doubles")
        self._ck(self._lib.rmhd2d_set_eta_table(self._h, a.ctypes.data_as(_DP)))

    def apply_boundary(self) -> None:
        self._ck(self._lib.rmhd2d_apply_boundary(self._h))

    # -- stepping --
    def calculate_dt(self) -> float:
        d = ctypes.c_double()
        self._ck(self._lib.rmhd2d_calculate_dt(self._h, ctypes.byref(d)))
        return d.value

    def step(self) -> None:
        self._ck(self._lib.rmhd2d_step_rk2(self._h))

    def run(self, nsteps: int) -> None:
        self._ck(self._lib.rmhd2d_run(self._h, int(nsteps)))

    # -- discrete adjoint (frozen dt) --
    def run_fixed_dt(self, dts) -> None:
        """Steps with the given dts instead of the CFL dt."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        self._ck(self._lib.rmhd2d_run_fixed_dt(self._h, len(d), d.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def adjoint_forward(self, nsteps: int, checkpoint_interval: int = 0) -> None:
        """nsteps steps, recording the dts and sqrt(N) checkpoints for adjoint_backward
        (checkpoint_interval 0; a negative one keeps every step's states, and backward recomputes nothing)."""
        self._ck(self._lib.rmhd2d_adjoint_forward(self._h, int(nsteps), int(checkpoint_interval)))
        self._adj_steps = int(nsteps)

    def adjoint_dts(self) -> np.ndarray:
        out = np.empty(getattr(self, "_adj_steps", 0), dtype=np.float64)
        self._ck(self._lib.rmhd2d_adjoint_dts(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def adjoint_backward(self, seed: np.ndarray, want_eta: bool = True):
        """(dJ/dU_0, dJ/d eta) for the seed dJ/dU_N of the recorded run."""
        sd = _as_f64(seed)
        if sd.size != self.nx * self.ny * 8:
            raise ValueError("seed must hold nx*ny*8 doubles")
        gs = np.empty((self.nx, self.ny, 8), dtype=np.float64)
        ge = np.empty((self.nx, self.ny), dtype=np.float64) if want_eta else None
        P = ctypes.POINTER(ctypes.c_double)
        self._ck(self._lib.rmhd2d_adjoint_backward(self._h, sd.ctypes.data_as(P), gs.ctypes.data_as(P),
                                                   ge.ctypes.data_as(P) if ge is not None else None))
        return gs, ge

    def adjoint_release(self) -> None:
        self._ck(self._lib.rmhd2d_adjoint_release(self._h))

    def set_tile_shape(self, shape: int) -> None:
        self._ck(self._lib.rmhd2d_set_tile_shape(self._h, int(shape)))

    @property
    def tile_shape(self) -> int:
        v = ctypes.c_int()
        self._ck(self._lib.rmhd2d_get_tile_shape(self._h, ctypes.byref(v)))
        return v.value

    def autotune(self, trial_steps: int = 4) -> int:
        """Times each tile shape (state restored) and keeps the fastest."""
        v = ctypes.c_int()
        self._ck(self._lib.rmhd2d_autotune(self._h, int(trial_steps), ctypes.byref(v)))
        return v.value

    def tuning(self) -> dict[int, tuple[float, float]]:
        """Tile shape -> (stage-1 ms, stage-2 ms) measured by the last autotune."""
        n = ctypes.c_int()
        sh = (ctypes.c_int * 8)()
        m1, m2 = (ctypes.c_float * 8)(), (ctypes.c_float * 8)()
        self._ck(self._lib.rmhd2d_get_tuning(self._h, 8, ctypes.byref(n), sh, m1, m2))
        return {int(sh[q]): (float(m1[q]), float(m2[q])) for q in range(min(n.value, 8))}

    @property
    def stage_shapes(self) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        self._ck(self._lib.rmhd2d_get_stage_shapes(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_stage_shapes(self, shape1: int, shape2: int) -> None:
        self._ck(self._lib.rmhd2d_set_stage_shapes(self._h, int(shape1), int(shape2)))

    def run_timed(self, nsteps: int) -> float:
        """run(nsteps) timed with CUDA events on the solver's stream; ms."""
        ms = ctypes.c_float()
        self._ck(self._lib.rmhd2d_run_timed(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def profile_step(self) -> list[float]:
        """One step; device ms of [stage 1, boundary, stage 2, boundary+CFL]."""
        ms = (ctypes.c_float * 4)()
        self._ck(self._lib.rmhd2d_profile_step(self._h, ms))
        return [float(v) for v in ms]

    @property
    def dt(self) -> float:
        d = ctypes.c_double()
        self._ck(self._lib.rmhd2d_get_dt(self._h, ctypes.byref(d)))
        return d.value

    @property
    def total_time(self) -> float:
        d = ctypes.c_double()
        self._ck(self._lib.rmhd2d_get_total_time(self._h, ctypes.byref(d)))
        return d.value

    def check_crashed(self) -> bool:
        c = ctypes.c_int()
        self._ck(self._lib.rmhd2d_check_crashed(self._h, ctypes.byref(c)))
        return bool(c.value)

    # -- snapshots --
    def save(self, directory: str, name_without_step: str, step: int) -> str:
        self._ck(self._lib.rmhd2d_save(self._h, os.fsencode(directory), os.fsencode(name_without_step), int(step)))
        return os.path.join(directory, f"{name_without_step}_{step}.bin")

    def load(self, path: str) -> None:
        self._ck(self._lib.rmhd2d_load(self._h, os.fsencode(path)))


class Batch:
    """Independent runs (own grid size, eta, walls) stepped together: each
    RK2 stage of all runs is one persistent launch over all their tiles,
    replayed from a CUDA graph.  ``batch[r]`` is a (non-owning) Solver view of
    run r for its state, eta table, dt, crash flag and snapshots."""

    def __init__(self, setups, precision: str = "fp64_exact", device: int = 0, apply_boundary: bool = True):
        lib = _lib.load()
        cfgs = (_lib.Config * len(setups))()
        for r, s in enumerate(setups):
            cfgs[r] = Solver.make_config(s.nx, s.ny, s.dx, s.dy, gamma=s.gamma, cfl=s.cfl, eps=s.eps, eta=s.eta,
                                         bc=s.bc, bc_y=s.bc_y, precision=precision, device=device,
                                         ct=getattr(s, "ct", "stage1"))
        h = ctypes.c_void_p()
        _lib.check_batch(lib.rmhd2d_batch_create(cfgs, len(setups), ctypes.byref(h)), None)
        self._lib, self._h = lib, h
        self.members = []
        for r, s in enumerate(setups):
            mh = ctypes.c_void_p()
            self._ck(lib.rmhd2d_batch_member(h, r, ctypes.byref(mh)))
            m = Solver._member(mh, s.nx, s.ny)
            if s.eta_table is not None:
                m.set_eta_table(s.eta_table)
            m.set_state(s.state, apply_boundary=apply_boundary)
            self.members.append(m)

    def _ck(self, st: int) -> None:
        _lib.check_batch(st, self._h)

    def __len__(self) -> int:
        return len(self.members)

    def __getitem__(self, r: int) -> Solver:
        mh = ctypes.c_void_p()
        self._ck(self._lib.rmhd2d_batch_member(self._h, int(r), ctypes.byref(mh)))
        return self.members[r]

    def run(self, nsteps: int) -> None:
        self._ck(self._lib.rmhd2d_batch_run(self._h, int(nsteps)))

    def run_timed(self, nsteps: int) -> float:
        ms = ctypes.c_float()
        self._ck(self._lib.rmhd2d_batch_run_timed(self._h, int(nsteps), ctypes.byref(ms)))
        return ms.value

    def set_launch(self, shape: int, ctas_per_sm: int) -> None:
        self._ck(self._lib.rmhd2d_batch_set_launch(self._h, int(shape), int(ctas_per_sm)))

    @property
    def launch(self) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        self._ck(self._lib.rmhd2d_batch_get_launch(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def autotune(self, trial_steps: int = 4) -> tuple[int, int]:
        a, b = ctypes.c_int(), ctypes.c_int()
        self._ck(self._lib.rmhd2d_batch_autotune(self._h, int(trial_steps), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def tuning(self) -> list[tuple[int, int, float]]:
        """(tile shape, CTAs per SM, ms per step) of each point the last autotune tried."""
        n = ctypes.c_int()
        sh, ct = (ctypes.c_int * 16)(), (ctypes.c_int * 16)()
        ms = (ctypes.c_float * 16)()
        self._ck(self._lib.rmhd2d_batch_get_tuning(self._h, 16, ctypes.byref(n), sh, ct, ms))
        return [(int(sh[q]), int(ct[q]), float(ms[q])) for q in range(min(n.value, 16))]

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            for m in self.members:
                m._h = ctypes.c_void_p()
            self._lib.rmhd2d_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def write_snapshot(path: str, state: np.ndarray) -> None:
    """Write a host state in the reference save() format (no GPU needed)."""
    lib = _lib.load()
    a = _as_f64(state)
    if a.ndim != 3 or a.shape[2] != 8:
        raise ValueError("state must have shape (nx, ny, 8)")
    _lib.check(lib.rmhd2d_write_snapshot(os.fsencode(path), a.ctypes.data_as(_DP), a.shape[0], a.shape[1]), None)


def read_snapshot(path: str, nx: int, ny: int) -> np.ndarray:
    """Read a save() file (the reference's or this library's)."""
    a = np.fromfile(path, dtype="<f8")
    if a.size != nx * ny * 8:
        raise ValueError(f"{path}: expected {nx * ny * 8} doubles, found {a.size}")
    return a.reshape(nx, ny, 8)


class ResistiveMHD2D:
    """Drop-in mirror of the reference's ``ResistiveMHD2D`` class.

    Subclass and override ``initializeU`` to fill ``self.U`` (an (nx, ny, 8)
    array, ghosts included) exactly as the reference's drivers implement
    ``ResistiveMHD2D::initializeU`` -- the boundary is applied afterwards,
    as those drivers do.  ``dt`` and ``totalTime`` mirror the reference's
    globals (const.hpp:20-23)."""

    def __init__(self, nx: int, ny: int, dx: float, dy: float, *, gamma_mhd: float = 5.0 / 3.0, CFL: float = 0.4,
                 EPS: float = 1e-20, eta: float = 0.0, boundary: str = "periodic", boundary_y: str | None = None,
                 eta_table=None, precision: str = "fp64_exact", device: int = 0, ct: str = "stage1"):
        self._s = Solver(nx, ny, dx, dy, gamma=gamma_mhd, cfl=CFL, eps=EPS, eta=eta, bc=boundary, bc_y=boundary_y,
                         precision=precision, device=device, ct=ct)
        if eta_table is not None:
            self._s.set_eta_table(eta_table)
        self.nx, self.ny = nx, ny
        self.U = np.zeros((nx, ny, 8), dtype=np.float64)
        self.dt = 0.0
        self.totalTime = 0.0

    @property
    def solver(self) -> Solver:
        return self._s

    def close(self) -> None:
        """Releases the device state now (the reference frees it in its destructor)."""
        self._s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def initializeU(self) -> None:
        """Override: fill self.U.  The default uploads self.U as it is."""

    def _upload(self) -> None:
        self._s.set_state(self.U, apply_boundary=True)

    def initialize(self) -> None:
        self.initializeU()
        self._upload()

    def oneStepRK2(self) -> None:
        """One RK2 step with the configured walls (the reference's oneStepRK2,
        or oneStepRK2PeriodicXSymmetricY with boundary='periodic',
        boundary_y='symmetric')."""
        self._s.step()
        self.dt = self._s.dt
        self.totalTime = self._s.total_time

    def calculateDt(self) -> float:
        self.dt = self._s.calculate_dt()
        return self.dt

    def checkCalculationIsCrashed(self) -> bool:
        return self._s.check_crashed()

    def getU(self) -> np.ndarray:
        return self._s.get_state()

    def save(self, directoryname: str, filenameWithoutStep: str, step: int) -> str:
        return self._s.save(directoryname, filenameWithoutStep, step)
