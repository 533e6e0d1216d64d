"""gravlume_b200: B200-native (sm_100a) Kerr-Newman null-geodesic tracing for Gravlume.

The product is libglc.so (gravlume_b200/_lib/, C ABI in include/glc.h): hand-written CUDA kernels
integrating the Hamiltonian null-geodesic system in Cartesian Kerr-Schild coordinates with an
adaptive Dormand-Prince 5(4) stepper in FP32, MIXED or FP64 precision. This package is the Python
host binding over that C ABI.
"""

from ._native import RESULT_FIELDS, GlcError, lib  # noqa: F401
from .batches import TileRegion, TraceProgress, tile_grid  # noqa: F401
from .build import LIB_PATH, build  # noqa: F401
from .trace import (  # noqa: F401
    EquatorialSurface, FootprintStatus, Graph, KerrSchildChart, Observation, Precision, ReferencePolicy, Termination,
    Tape, TracePipeline, TraceResults, footprint_fields, image_camera, oblate_to_cartesian, prograde_isco, raylist_camera,
)
