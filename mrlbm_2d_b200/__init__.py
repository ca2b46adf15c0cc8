"""B200-native moment-regularized D2Q9 cylinder-flow step (drop-in for mrlbm_2d's hot path).

`Config` mirrors the reference's input.dat namelists; `Simulation` drives one case through
the C ABI of libmrlbm.so (include/mrlbm.h).  The CUDA library is required: there is no CPU
fallback.
"""
from .config import Config  # noqa: F401
from .api import (BATCH_GRAPH, BATCH_PERSISTENT, BATCH_STREAMS, FP32, FP64, N_TILE_CONFIGS, Batch, MrlbmError, Simulation, config_from_namelist, cp_statistics,  # noqa: F401
                  force_statistics, load_library, rho_inlet_running_mean, slabs_step)
