"""The low-level module of the mirror, as ``within._within`` is for within-py: the same
classes and functions, including the local-solver configuration classes that the
reference exposes only here (``ApproxCholConfig``, ``ApproxSchurConfig``,
``SchurComplement``)."""
from . import (  # noqa: F401
    CG,
    GMRES,
    LSMR,
    AdditiveSchwarz,
    AdditiveSchwarzDiagnostics,
    ApproxCholConfig,
    ApproxSchurConfig,
    BatchSolveResult,
    FePreconditioner,
    MultiplicativeSchwarz,
    OperatorRepr,
    Preconditioner,
    ReductionStrategy,
    SchurComplement,
    SolveResult,
    Solver,
    solve,
    solve_batch,
)
