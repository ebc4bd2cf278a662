"""B200-native MAS-preconditioned PCG for StiffGIPC's Newton-step linear solve.

``solver.MasPcg`` is the entry point; ``include/maspcg.h`` is the C ABI it
binds; ``synth`` builds the seeded benchmark systems.
"""
from .solver import MasPcg, PCGSolver, PCGSolverConfig, TraditionalMAS32Preconditioner  # noqa: F401
