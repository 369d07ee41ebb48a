"""bowshock_b200: bowshock's steady 2D axisymmetric Euler solve on NVIDIA B200.

The solver runs as hand-written sm_100a CUDA kernels inside
`lib/libbowshock_b200.so`, reached through the C ABI of include/bowshock.h.
There is no CPU fallback: creating an engine without the built library or
without a GPU raises.
"""
from .config import (  # noqa: F401
    Boundary,
    Euler2DConfig,
    FreeStream,
    Primitive2D,
    StructuredGrid,
    free_stream_at,
    fround,
    grid_from_function,
    rectangular_grid,
    steady_drag_config,
)

__version__ = "0.1.0"
