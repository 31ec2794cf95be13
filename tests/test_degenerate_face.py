"""The HLLD degenerate case the reference does not guard.

tests/golden/plasmoid_degenerate_face.npz holds a 20 x 20 window of the
8192 x 4096 plasmoid-unstable sheet one step before the run in the
reference's arithmetic first produces a NaN energy (step 934), and that
step's dt (made by make_plasmoid_degenerate_face.py).  At its centre an
x-face's star denominator rho (S - u)(S - SM) - bX^2 rounds to exactly 0
(the fast and Alfven waves meet where |bY| ~ 1e-4); the reference adds only
EPS = 1e-20, so v*, bY* and the double-star state built from them blow up,
and the face's flux is enough to wreck the next step.  One step of the
window with periodic walls reproduces it: the edge cells see the wrap, the
centre does not.

* the oracle turns the same three cells non-finite (the claim is the
  reference's, not this build's);
* the drop-in (fp64_exact) matches the oracle bit for bit there and
  everywhere else at the centre;
* fp64_fast (its rearranged denominators do not cancel to 0 here) and
  fp32_bulk (which takes the degenerate branch below 1e-5 bX^2) stay finite."""
from pathlib import Path

import numpy as np
import pytest

FIXTURE = Path(__file__).parent / "golden" / "plasmoid_degenerate_face.npz"
CENTRE = (slice(6, 14), slice(6, 14))   # cells the periodic wrap cannot reach in one step


def _window():
    from resistivemhd_gpu_b200.setups import Setup

    d = np.load(FIXTURE)
    w = d["window"]
    s = Setup("plasmoid_window", w.copy(), float(d["dx"]), float(d["dy"]), float(d["gamma"]), 0.4, 1e-20,
              float(d["eta"]), None, "periodic")
    return s, float(d["dt"]), [tuple(c) for c in d["nonfinite"].tolist()]


def _oracle_step():
    from oracle.oracle import TangentLib

    s, dt, bad = _window()
    out = TangentLib().run_fixed_dt(s, s.state, np.array([dt]), apply_boundary=False)
    return (out[0] if isinstance(out, tuple) else out), bad


def test_oracle_reproduces_the_reference_nan():
    out, bad = _oracle_step()
    got = sorted(map(tuple, np.argwhere(~np.isfinite(out[..., 7])).tolist()))
    assert got == sorted(bad) == [(10, 10), (10, 11), (11, 10)]


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64_exact", "fp64_fast", "fp32_bulk"])
def test_degenerate_face_on_the_gpu(gpu, precision):
    from resistivemhd_gpu_b200 import Solver

    s, dt, bad = _window()
    want, _ = _oracle_step()
    with Solver.from_setup(s, precision=precision, apply_boundary=False) as sol:
        sol.run_fixed_dt([dt])
        got = sol.get_state()
    c = got[CENTRE]
    if precision == "fp64_exact":
        assert np.array_equal(c, want[CENTRE], equal_nan=True)
        assert sorted(map(tuple, np.argwhere(~np.isfinite(got[..., 7])).tolist())) == sorted(bad)
    else:
        assert np.isfinite(c).all()
        # the smooth start (|v| ~ 1e-4, rho ~ 0.1, |B| ~ 1) moves by a small
        # fraction in one step where the face stays bounded
        rel = np.abs(c[..., 7] - s.state[CENTRE][..., 7]) / np.abs(s.state[CENTRE][..., 7])
        assert rel.max() < 1e-2, rel.max()
