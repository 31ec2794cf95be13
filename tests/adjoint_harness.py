"""Gradient-check harness for the discrete adjoint: a torch.autograd.Function
over the C-ABI forward/backward pair, so a misfit written in torch
differentiates through the solver.  Test infrastructure only."""
import numpy as np
import torch


class FrozenDtRun(torch.autograd.Function):
    """U_N = run(U_0, eta) for `nsteps` steps of a periodic solver, dt of each
    step recorded on the forward pass and held fixed for the gradient."""

    @staticmethod
    def forward(ctx, state0, eta, solver, nsteps, interval):
        solver.set_eta_table(eta.detach().cpu().numpy())
        solver.set_state(state0.detach().cpu().numpy(), apply_boundary=True)
        solver.adjoint_forward(nsteps, interval)
        ctx.solver = solver
        return torch.from_numpy(solver.get_state().copy())

    @staticmethod
    def backward(ctx, grad_out):
        gs, ge = ctx.solver.adjoint_backward(grad_out.detach().cpu().numpy().astype(np.float64))
        return torch.from_numpy(gs), torch.from_numpy(ge), None, None, None


MISFIT_FIELDS = (0, 4, 5, 6)   # rho, bX, bY, bZ


def misfit(final, target):
    """L2 misfit of the interior (rho, bX, bY, bZ) of the final state."""
    d = final[3:-3, 3:-3, list(MISFIT_FIELDS)] - target[3:-3, 3:-3, list(MISFIT_FIELDS)]
    return 0.5 * (d * d).sum()


def misfit_difference(final_p: np.ndarray, final_m: np.ndarray, target: np.ndarray) -> float:
    """misfit(final_p) - misfit(final_m), formed as sum (f_p - f_m) (mean -
    target): the same number without subtracting two large misfits, whose
    own rounding would swamp a central difference along a localized
    direction."""
    f = list(MISFIT_FIELDS)
    fp, fm, t = final_p[3:-3, 3:-3, f], final_m[3:-3, 3:-3, f], target[3:-3, 3:-3, f]
    return float(((fp - fm) * (0.5 * (fp + fm) - t)).sum())


def misfit_seed(final: np.ndarray, target: np.ndarray) -> np.ndarray:
    seed = np.zeros_like(final)
    f = list(MISFIT_FIELDS)
    seed[3:-3, 3:-3, f] = final[3:-3, 3:-3, f] - target[3:-3, 3:-3, f]
    return seed
