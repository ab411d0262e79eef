"""B200-native Barnes-Hut engine for the per-step compute pipeline of the
ElliottF05/webgpu-fluid-sim N-body simulator.

The package directory name has hyphens, so load it with
``importlib.import_module("webgpu-fluid-sim_b200")`` after putting the
repository root on ``sys.path``.
"""
from ._lib import (BH_DEBUG_LOOKBACK_UNPUBLISHED, BH_DEBUG_SPLIT_BUILD,  # noqa: F401
                   BH_ERR_DEVICE_CHECK, BH_OK, BhError, load)
from .config import WORKLOADS, Config, getDefaultConfig  # noqa: F401
from .render import RenderCommand, Renderer  # noqa: F401
from .runlog import RunLog  # noqa: F401
from .shard import (ShardedSimulation, all_gather_chunks, chunk_bytes,  # noqa: F401
                    chunk_capacity, partition_systems, slot_ranges)
from .simulation import (SCENARIOS, CommandBuffer, Ensemble, SimBuffers,  # noqa: F401
                         Simulation, ensemble_sizes, generate_scenario, submit)
