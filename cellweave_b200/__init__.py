"""cellweave_b200: cellweave's per-step hot path on one B200 (sm_100a).

The CPM Metropolis sweep, the red-black SOR field solve and the per-cell RK4
network step of ngodzik/cellweave's engine crate, as CUDA kernels behind the
C ABI of ``include/cellweave_b200.h``; ``engine`` mirrors the engine crate's
API over it.  There is no CPU path: without the built library or a GPU every
compute call raises.
"""
from ._lib import (CellweaveError, ConfigError, CudaError, NotFoundError, OdeSolverError,  # noqa: F401
                   SimulationError)
from .engine import (FP32_DC, FP64, LIN_SINK, OBSTACLE, PRODUCTION, UPTAKE, VALUES, WINDOW_64, WINDOW_AUTO, WINDOW_TALL, STOP_MAX_CHANGE, STOP_RESIDUAL, CpmLattice, Fit, Network,  # noqa: F401
                     ScalarField, Simulation, apply_background_uptake, apply_production, apply_uptake,
                     hold_medium_bath, hold_obstacles_at, load_network_spec, mean_per_cell)
from . import config, output  # noqa: F401,E402
