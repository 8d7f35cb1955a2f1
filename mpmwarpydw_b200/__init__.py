"""mpmwarpydw_b200: B200 (sm_100a) implementation of the MPMWarpYDW MPM-XPBD substep.

Compute runs in libmpmw.so (hand-written CUDA, C ABI in include/mpmw.h);
PyTorch owns device memory and streams.  ``mpmwarpydw_b200.utils`` mirrors the
reference's ``utils`` package (mpmRoutines, mpmRoutinesDruckerPrager,
xpbdRoutines, simulationRoutines, simStates, getArgs).
"""
__version__ = "0.1.0"
