"""B200-native (sm_100a) 2D resistive-MHD RK2 step.

A drop-in for the single-GPU Thrust library of keita-akutagawa/ResistiveMHD_GPU
(HLLD fluxes, MUSCL-minmod reconstruction, constrained transport, eta*J
resistive term, Heun RK2 with a fused CFL reduction), exposed through the C
ABI in include/rmhd2d.h (librmhd2d.so, built in this directory) and the
Python mirror below.
"""
from .solver import Batch, ResistiveMHD2D, Solver, read_snapshot, write_snapshot  # noqa: F401
from . import setups  # noqa: F401

__all__ = ["Batch", "ResistiveMHD2D", "Solver", "read_snapshot", "write_snapshot", "setups"]
