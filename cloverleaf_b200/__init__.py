"""B200-native backend for the CloverLeaf hydro path.

The product is libcloverb200.so (CUDA kernels for sm_100a behind the C ABI in
include/cloverb200.h) and the C++ model glue in cloverleaf_b200/model/ that
lets the reference's unchanged driver run on it.  This package adds a ctypes
binding (`Chunk`), the driver's call sequence in Python (`HydroRun`) and a
deck reader, for tests and benchmarks.
"""
from .chunk import (FIELD_ID, FIELD_NAMES, FP32, FP64, GEOM_ID, GEOM_NAMES, Chunk, CloverError,  # noqa: F401
                    library)
from .deck import Deck, State, benchmark_deck, format_deck, nudged, parse_deck, read_deck  # noqa: F401
from .hydro import HydroRun, Summary  # noqa: F401
from .batch import Batch, ensemble_deck, ensemble_decks  # noqa: F401
from .adjoint import Adjoint, kinetic_energy_function  # noqa: F401
