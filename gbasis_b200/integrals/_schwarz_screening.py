"""``gbasis.integrals._schwarz_screening`` (``_schwarz_screening.py:14-218``) on the engine."""
from ..schwarz_screening import (  # noqa: F401
    SchwarzScreener,
    compute_schwarz_bound_shell_pair,
    compute_schwarz_bounds,
    shell_pair_significant,
)

__all__ = ["compute_schwarz_bound_shell_pair", "compute_schwarz_bounds",
           "shell_pair_significant", "SchwarzScreener"]
