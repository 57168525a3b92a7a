"""a5_streamer_b200: B200-native (sm_100a) rebuild of a5_streamer's per-timestep
hot path (Koren drift-diffusion fluxes and source update, transport lookups,
space charge, FAS multigrid Poisson solve and field from potential) on an
Afivo quadtree, behind a C ABI (include/a5g.h)."""
from . import config  # noqa: F401

__all__ = ["config"]
