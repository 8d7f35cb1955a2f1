"""Reference-named modules of the MPM-XPBD substep (drop-in for MPMWarpYDW ``utils``)."""
