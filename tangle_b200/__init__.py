"""tangle_b200: TANGLE's plain relaxation path on NVIDIA B200 (sm_100a).

The "cuda" backend of the reference's relaxation seam: the uniform-grid cell
list, Verlet neighbor lists, capsule contact projection, stretch /
rest-shape bend / admissible-curvature projections and the overlap and
curvature reductions, as hand-written CUDA kernels behind the C ABI of
include/tangle_cuda.h, with the reference's Python surface
(`RelaxationSettings`, `Recipe.run`, `RunResult`) on top, and the formation
hooks of the resident world (staged activation, layer and vertex targets,
cell compaction and its metrics).
"""

from .assembly import Cell, FiberAssembly, Material, PackedAssembly
from .device import DeviceWorld, load_library
from .formation import (CompactionEnergyModel, CompactionKinematics, CompactionMetrics, FormationTargetError)
from .generate import FiberPopulation, SplitMix64, generate_fiber_population
from .recipe import FiberSelection, HeldTargets, Recipe, RecipeError, RunResult
from .settings import BatchStatus, CellListConfig, RelaxationConfig, RelaxationSettings

__all__ = [
    "BatchStatus", "Cell", "CellListConfig", "CompactionEnergyModel", "CompactionKinematics", "CompactionMetrics",
    "DeviceWorld", "FiberAssembly", "FiberPopulation", "FiberSelection", "FormationTargetError", "HeldTargets",
    "Material", "PackedAssembly", "Recipe", "RecipeError", "RelaxationConfig", "RelaxationSettings", "RunResult",
    "SplitMix64", "generate_fiber_population", "load_library",
]
