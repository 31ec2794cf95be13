"""Seeded initial states for the benchmark and test configurations.

Every state is returned in the reference's layout: a float64 array of shape
``(nx, ny, 8)`` with fields ``rho, rhoU, rhoV, rhoW, bX, bY, bZ, e`` (cell
``k = j + i*ny`` of the reference's flat array is ``state[i, j]``).  ``nx``
and ``ny`` include 3 ghost layers per side, as the reference's do
(lib_ResistiveMHD_2D_GPU_periodicXY/boundary.cu:9-57 copies cells
``nx-6..nx-4`` into ``0..2``), so a config of N x M cells has
``nx, ny = N + 6, M + 6``.

Conventions (the same on the oracle and CUDA sides):

* physical cell ``i`` has centre ``x_i = xmin + (i - 3 + 1/2) dx``;
* ``bX[i, j]`` is the x-face value at ``x_{i+1/2}``, ``bY[i, j]`` the y-face
  value at ``y_{j+1/2}`` (reference
  ``shiftBXToCenterForCT_kernel``, resistiveMHD_2D.cu:313-324);
* where a flux function A_z is given, face B is its discrete curl on cell
  corners, so the discrete div B is zero to round-off;
* noise is drawn from a counter-based generator (splitmix64) keyed by
  ``(seed, field, i, j)``, so a state does not depend on array order;
* the state is filled everywhere, ghosts included; callers then apply the
  boundary (the reference's drivers do the same in ``initializeU``).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

GHOST = 3
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & _M64
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M64
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M64
    return z ^ (z >> np.uint64(31))


def uniform_noise(seed: int, field: int, nx: int, ny: int) -> np.ndarray:
    """Uniform values in [-1, 1) keyed by (seed, field, i, j)."""
    i = np.arange(nx, dtype=np.uint64)[:, None]
    j = np.arange(ny, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        key = (np.uint64(seed) * np.uint64(0xD1B54A32D192ED03)
               + np.uint64(field) * np.uint64(0x8CB92BA72F3D8DD7)
               + i * np.uint64(0x9E3779B97F4A7C15) + j * np.uint64(0xC2B2AE3D27D4EB4F)) & _M64
        h = _splitmix64(_splitmix64(key))
    return (h >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


@dataclasses.dataclass
class Setup:
    """An initial state plus the solver parameters it is meant for."""
    name: str
    state: np.ndarray            # (nx, ny, 8) float64
    dx: float
    dy: float
    gamma: float
    cfl: float
    eps: float
    eta: float                   # scalar eta (uniform resistivity and the dt limit)
    eta_table: np.ndarray | None  # (nx, ny) cell-centred eta, or None for uniform
    bc: str                      # x walls: "periodic" or "symmetric"
    xmin: float = 0.0
    ymin: float = 0.0
    bc_y: str | None = None      # y walls, None for the same as bc
    ct: str = "stage1"           # "stage1": CT with the stage-1 EMF; "contact": CT-Contact EMF

    @property
    def nx(self) -> int:
        return self.state.shape[0]

    @property
    def ny(self) -> int:
        return self.state.shape[1]

    @property
    def interior_cells(self) -> int:
        return (self.nx - 2 * GHOST) * (self.ny - 2 * GHOST)


def _centres(n: int, lo: float, d: float) -> np.ndarray:
    return lo + (np.arange(n) - GHOST + 0.5) * d


def _faces(n: int, lo: float, d: float) -> np.ndarray:
    return lo + (np.arange(n) - GHOST + 1.0) * d


def _energy(rho, u, v, w, bxc, byc, bz, p, gamma):
    return p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w) + 0.5 * (bxc * bxc + byc * byc + bz * bz)


def _pack(rho, u, v, w, bx, by, bz, e) -> np.ndarray:
    s = np.empty(rho.shape + (8,), dtype=np.float64)
    s[..., 0] = rho
    s[..., 1] = rho * u
    s[..., 2] = rho * v
    s[..., 3] = rho * w
    s[..., 4] = bx
    s[..., 5] = by
    s[..., 6] = bz
    s[..., 7] = e
    return s


def orszag_tang(n: int = 256, m: int | None = None, eta: float = 1e-3, noise: float = 1e-6,
                seed: int = 1, cfl: float = 0.4, gamma: float = 5.0 / 3.0) -> Setup:
    """Orszag-Tang vortex on [0, 2pi)^2, periodic: rho = gamma^2, p = gamma,
    vx = -sin y, vy = sin x, Bx = -sin y, By = sin 2x, vz = Bz = 0, plus
    uniform noise of amplitude ``noise`` on vx and vy."""
    m = n if m is None else m
    nx, ny = n + 2 * GHOST, m + 2 * GHOST
    dx, dy = 2.0 * math.pi / n, 2.0 * math.pi / m
    xc, yc = _centres(nx, 0.0, dx)[:, None], _centres(ny, 0.0, dy)[None, :]
    shape = (nx, ny)
    rho = np.full(shape, gamma * gamma)
    p = np.full(shape, gamma)
    u = -np.sin(yc) + noise * uniform_noise(seed, 1, nx, ny)
    v = np.sin(xc) + noise * uniform_noise(seed, 2, nx, ny)
    w = np.zeros(shape)
    # Bx depends on y only and By on x only, so point values on the faces
    # are exactly divergence free.
    bx = np.broadcast_to(-np.sin(yc), shape).copy()
    by = np.broadcast_to(np.sin(2.0 * xc), shape).copy()
    bz = np.zeros(shape)
    e = _energy(rho, u, v, w, bx, by, bz, p, gamma)
    return Setup("orszag_tang", _pack(rho, u, v, w, bx, by, bz, e), dx, dy, gamma, cfl, 1e-20,
                 eta, None, "periodic")


def harris_sheet(n: int = 2048, m: int = 1024, xlen: float = 128.0, ylen: float = 64.0,
                 width: float = 0.5, beta: float = 0.2, psi0: float = 0.03, noise: float = 1e-3,
                 eta0: float = 1e-3, eta_bump: float = 1e-2, bump_width: float = 1.0,
                 seed: int = 2, cfl: float = 0.4, gamma: float = 5.0 / 3.0,
                 name: str = "harris") -> Setup:
    """Harris current sheet on [-xlen/2, xlen/2] x [-ylen/2, ylen/2], symmetric
    boundaries.  Bx = tanh(y/width) + perturbation, rho = sech^2(y/width) +
    beta, p = (beta + sech^2(y/width)) / 2 (pressure balance for B0 = 1, so
    beta is the upstream plasma beta).  The flux-function perturbation
    psi = psi0 cos(2 pi x / xlen) cos(pi y / ylen) is added to the base flux
    function width * ln cosh(y/width) and the face B is the discrete curl of
    their sum on cell corners.  eta = eta0 + eta_bump exp(-r^2 / bump_width^2)
    is tabulated at cell centres; the dt limit uses its maximum."""
    nx, ny = n + 2 * GHOST, m + 2 * GHOST
    xmin, ymin = -0.5 * xlen, -0.5 * ylen
    dx, dy = xlen / n, ylen / m
    xc, yc = _centres(nx, xmin, dx)[:, None], _centres(ny, ymin, dy)[None, :]
    xf, yf = _faces(nx, xmin, dx), _faces(ny, ymin, dy)

    def az(x, y):
        return width * np.log(np.cosh(y / width)) + psi0 * np.cos(2.0 * math.pi * x / xlen) * np.cos(math.pi * y / ylen)

    # corner values A(x_{i+1/2}, y_{j+1/2}) for i, j in [-1, n) so that faces
    # of every cell have both corners.
    xcor = np.concatenate([[xf[0] - dx], xf])[:, None]
    ycor = np.concatenate([[yf[0] - dy], yf])[None, :]
    A = az(xcor, ycor)                        # (nx+1, ny+1): A[i+1, j+1] = corner (i+1/2, j+1/2)
    bx = (A[1:, 1:] - A[1:, :-1]) / dy        # x-face (i+1/2, j)
    by = -(A[1:, 1:] - A[:-1, 1:]) / dx       # y-face (i, j+1/2)
    sech2 = 1.0 / np.cosh(yc / width) ** 2
    shape = (nx, ny)
    rho = np.broadcast_to(sech2 + beta, shape).copy()
    p = np.broadcast_to(0.5 * (beta + sech2), shape).copy()
    u = noise * uniform_noise(seed, 1, nx, ny)
    v = noise * uniform_noise(seed, 2, nx, ny)
    w = np.zeros(shape)
    bz = np.zeros(shape)
    bxc = 0.5 * (bx + np.concatenate([bx[:1], bx[:-1]], axis=0))
    byc = 0.5 * (by + np.concatenate([by[:, :1], by[:, :-1]], axis=1))
    e = _energy(rho, u, v, w, bxc, byc, bz, p, gamma)
    eta_tab = eta0 + eta_bump * np.exp(-(xc * xc + yc * yc) / (bump_width * bump_width))
    eta_tab = np.ascontiguousarray(np.broadcast_to(eta_tab, shape), dtype=np.float64)
    return Setup(name, _pack(rho, u, v, w, bx, by, bz, e), dx, dy, gamma, cfl, 1e-20,
                 float(eta0 + eta_bump), eta_tab, "symmetric", xmin, ymin)


def plasmoid_sheet(n: int = 8192, m: int = 4096, **kw) -> Setup:
    """Thin sheet (half-width 0.1, beta 0.1, uniform eta 1e-5), otherwise the
    Harris set-up; white-noise velocity perturbation of amplitude 1e-4."""
    s = harris_sheet(n, m, width=0.1, beta=0.1, noise=1e-4, eta0=1e-5, eta_bump=0.0, seed=3,
                     name="plasmoid", **kw)
    s.eta_table = None
    s.eta = 1e-5
    return s


def random_smooth_state(n: int, m: int, seed: int = 7, bc: str = "periodic", amp: float = 0.05,
                        eta: float = 2e-3, with_table: bool = False, gamma: float = 5.0 / 3.0,
                        bc_y: str | None = None) -> Setup:
    """Generic smooth, positive, divergence-free state for parity tests on
    small and ragged grids: every field varies in both directions and carries
    a little noise, so every branch of the solver is exercised."""
    nx, ny = n + 2 * GHOST, m + 2 * GHOST
    dx, dy = 1.0 / n, 1.3 / m
    xc, yc = _centres(nx, 0.0, dx)[:, None], _centres(ny, 0.0, dy)[None, :]
    xf, yf = _faces(nx, 0.0, dx), _faces(ny, 0.0, dy)
    tw = 2.0 * math.pi
    r = lambda f: uniform_noise(seed, f, nx, ny)
    rho = 1.0 + 0.3 * np.sin(tw * xc) * np.cos(tw * yc / 1.3) + amp * r(1) * 0.2
    p = 0.8 + 0.2 * np.cos(tw * (xc + yc / 1.3)) + amp * r(2) * 0.2
    u = 0.4 * np.sin(tw * yc / 1.3) + amp * r(3)
    v = -0.3 * np.sin(tw * xc) + amp * r(4)
    w = 0.2 * np.cos(tw * xc) * np.sin(tw * yc / 1.3) + amp * r(5)
    bz = 0.3 * np.cos(tw * (xc - yc / 1.3)) + amp * r(6)
    xcor = np.concatenate([[xf[0] - dx], xf])[:, None]
    ycor = np.concatenate([[yf[0] - dy], yf])[None, :]
    A = 0.15 * np.cos(tw * xcor) * np.cos(tw * ycor / 1.3) + 0.1 * np.sin(tw * (xcor + 2 * ycor / 1.3))
    A = A + 1e-3 * uniform_noise(seed, 9, nx + 1, ny + 1)
    bx = (A[1:, 1:] - A[1:, :-1]) / dy
    by = -(A[1:, 1:] - A[:-1, 1:]) / dx
    bxc = 0.5 * (bx + np.concatenate([bx[:1], bx[:-1]], axis=0))
    byc = 0.5 * (by + np.concatenate([by[:, :1], by[:, :-1]], axis=1))
    e = _energy(rho, u, v, w, bxc, byc, bz, p, gamma)
    tab = None
    if with_table:
        tab = np.ascontiguousarray(eta * (1.0 + 0.5 * np.sin(tw * xc) ** 2 * np.cos(tw * yc / 1.3) ** 2)
                                   * np.ones((nx, ny)))
    return Setup("random_smooth", _pack(rho, u, v, w, bx, by, bz, e), dx, dy, gamma, 0.4, 1e-20,
                 float(eta * 1.5) if with_table else eta, tab, bc, bc_y=bc_y)


def gaussian_random_field(n: int, m: int, lx: float, ly: float, corr: float, seed: int) -> np.ndarray:
    """Periodic Gaussian random field on an n x m cell-centred grid of a
    lx x ly box: white noise (Box-Muller on the counter-based generator)
    filtered in Fourier space by exp(-|k|^2 corr^2 / 4), the square root of
    the spectrum of the covariance exp(-r^2 / (2 corr^2)), then scaled to
    zero mean and unit variance."""
    u1 = 0.5 * (uniform_noise(seed, 101, n, m) + 1.0)
    u2 = 0.5 * (uniform_noise(seed, 102, n, m) + 1.0)
    white = np.sqrt(-2.0 * np.log(np.maximum(u1, 1e-300))) * np.cos(2.0 * math.pi * u2)
    kx = 2.0 * math.pi * np.fft.fftfreq(n, d=lx / n)[:, None]
    ky = 2.0 * math.pi * np.fft.fftfreq(m, d=ly / m)[None, :]
    g = np.real(np.fft.ifft2(np.fft.fft2(white) * np.exp(-(kx * kx + ky * ky) * corr * corr / 4.0)))
    g -= g.mean()
    return g / g.std()


def _periodic_extend(a: np.ndarray) -> np.ndarray:
    """Interior (n, m) array -> (n + 6, m + 6) with periodic ghosts."""
    return np.pad(a, GHOST, mode="wrap")


def ot_adjoint(n: int = 512, seed: int = 5, eta0: float = 1e-3, corr: float = 0.3, **kw) -> Setup:
    """Orszag-Tang vortex with a spatial resistivity eta = eta0 exp(g / 2),
    g a periodic Gaussian random field of correlation length `corr` (the
    inverse problem's parameter field), tabulated at cell centres; the dt
    limit uses the table's maximum."""
    s = orszag_tang(n, **kw)
    g = gaussian_random_field(n, n, 2.0 * math.pi, 2.0 * math.pi, corr, seed)
    tab = np.ascontiguousarray(_periodic_extend(eta0 * np.exp(0.5 * g)))
    s.name = "ot_adjoint"
    s.eta_table = tab
    s.eta = float(tab.max())
    return s


def kelvin_helmholtz(n: int = 256, m: int | None = None, width: float = 0.05, amp: float = 1e-2,
                     guide: float = 0.1, rho0: float = 1.0, p0: float = 1.0, eta: float = 1e-3,
                     seed: int = 4, cfl: float = 0.4, gamma: float = 5.0 / 3.0) -> Setup:
    """Periodic double shear layer on [0, 1)^2: vx = (tanh((y - 1/4)/w) -
    tanh((y - 3/4)/w) - 1) / 2 (two tanh layers, so the flow is periodic in
    y), vy = amp (sin(2 pi x) + noise) times Gaussians of width w about the
    layers, uniform rho = rho0 and p = p0, and an in-plane guide field
    Bx = guide along the flow (By = Bz = 0), uniform eta."""
    m = n if m is None else m
    nx, ny = n + 2 * GHOST, m + 2 * GHOST
    dx, dy = 1.0 / n, 1.0 / m
    xc, yc = _centres(nx, 0.0, dx)[:, None], _centres(ny, 0.0, dy)[None, :]
    shape = (nx, ny)
    # periodic images of the layer positions keep the ghosts consistent
    yw = np.mod(yc, 1.0)
    u = np.broadcast_to(0.5 * (np.tanh((yw - 0.25) / width) - np.tanh((yw - 0.75) / width) - 1.0), shape).copy()
    env = np.exp(-((yw - 0.25) ** 2) / (2 * width * width)) + np.exp(-((yw - 0.75) ** 2) / (2 * width * width))
    v = amp * (np.sin(2.0 * math.pi * xc) + uniform_noise(seed, 2, nx, ny)) * env
    rho = np.full(shape, rho0)
    p = np.full(shape, p0)
    w = np.zeros(shape)
    bx = np.full(shape, guide)
    by = np.zeros(shape)
    bz = np.zeros(shape)
    e = _energy(rho, u, v, w, bx, by, bz, p, gamma)
    return Setup("kelvin_helmholtz", _pack(rho, u, v, w, bx, by, bz, e), dx, dy, gamma, cfl, 1e-20, eta,
                 None, "periodic")


ENSEMBLE_SIZES = (128, 192, 256, 384, 512)


def ensemble(nruns: int = 256, seed: int = 4, eta_range: tuple[float, float] = (1e-4, 1e-2)) -> list[Setup]:
    """Independent periodic runs of uneven size: grid n x n with n drawn from
    ENSEMBLE_SIZES, eta log-uniform in eta_range, even runs Orszag-Tang and
    odd runs Kelvin-Helmholtz, all drawn from one seeded generator."""
    rng = np.random.default_rng(seed)
    sizes = rng.choice(ENSEMBLE_SIZES, size=nruns)
    etas = np.exp(rng.uniform(math.log(eta_range[0]), math.log(eta_range[1]), size=nruns))
    out = []
    for r in range(nruns):
        n, eta = int(sizes[r]), float(etas[r])
        s = orszag_tang(n, eta=eta, seed=1000 + r) if r % 2 == 0 else kelvin_helmholtz(n, eta=eta, seed=1000 + r)
        out.append(s)
    return out
