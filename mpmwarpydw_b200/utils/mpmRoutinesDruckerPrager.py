"""utils/mpmRoutinesDruckerPrager.py is empty in the reference (0 bytes); its
Drucker-Prager return map lives in utils/mpmRoutines.py:314-453.  This module
re-exports the stress kernels that run it so imports of either name work."""
from .mpmRoutines import (compute_stress_from_F_trial, drucker_prager_return_mapping,  # noqa: F401
                          kirchoff_stress)

__all__ = ["compute_stress_from_F_trial", "drucker_prager_return_mapping", "kirchoff_stress"]
