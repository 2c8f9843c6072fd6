"""cellshard_b200: B200-native (sm_100a) CellShard sparse execution hot path.

The compute lives in libcellshard_b200.so (hand-written CUDA behind a C ABI,
include/cellshard_b200.h).  This package holds the Python side of that
boundary: ctypes bindings (_abi), device-format helpers (device), the
mask_groups runtime mirror (runtime) and the synthetic data generator
(synth).  Importing it does not touch the GPU; the first call that needs the
library loads it and fails loudly if it has not been built.
"""

from ._abi import CellShardError, load  # noqa: F401

__all__ = ["CellShardError", "load"]
