"""B200-native RRTM longwave + shortwave column radiation (the WOOF-NAM radiation hot path).

Public API:
  RadSolver / SolverConfig   the library handle (woof_nam_b200.solver)
  make_columns               seeded synthetic column states (woof_nam_b200.columns)
  rrtm_call                  the reference's radiation-driver hook signature (woof_nam_b200.driver)
"""
from .columns import Columns, make_columns, workload  # noqa: F401


def __getattr__(name):
    if name in ("RadSolver", "SolverConfig"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
