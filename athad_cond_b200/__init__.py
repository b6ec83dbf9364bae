"""athad_cond_b200 - B200 (sm_100a) implementation of the ATHAD_COND model-iteration hot path.

The product is libathad_gpu.so (C ABI, include/athad_gpu.h).  This package holds its
CUDA sources (csrc/), the Python view of the ABI used by the tests and the benchmark, and
a seeded synthetic-state builder.  Importing the package does not require a GPU; creating a
GpuAtmosphere does, and fails loudly without one or without the built library.
"""
from ._abi import (FIELD, FIELD_NAMES, FIELD2D, PROFILE, InitConfig, Params, Precision, Status, Turb,  # noqa: F401
                   Wall, config_init, default_params, load_library, LIB_PATH)
from .context import AthadError, GpuAtmosphere, GpuBatch, default_init_config  # noqa: F401
from .synthetic import make_state, mirror, layer_heights  # noqa: F401

__all__ = ["GpuAtmosphere", "GpuBatch", "AthadError", "make_state", "mirror", "layer_heights",
           "default_params", "load_library", "Params", "FIELD", "FIELD_NAMES", "Turb", "Wall",
           "Precision", "InitConfig", "config_init", "default_init_config"]
