"""dba_b200 -- B200-native dynamic-block-activation (DBA) stencil engine.

Python view of the C ABI in include/dba.h (the library dba_b200/libdba_b200.so
built by dba_b200/build.py).  The engine runs only on the GPU; there is no CPU
fallback: importing works without a GPU, but creating a Simulation needs the
compiled library and a CUDA device.
"""
from .engine import (  # noqa: F401
    BATCH_PERSISTENT, BATCH_WAIT_LIMIT, DBA_ERR, FIELDS, MODELS, OPT_WAIT_LIMIT, Batch, Config, DBAError, Simulation,
    config, lib_path, load_library, parse_input,
)

__all__ = ["Batch", "Config", "DBAError", "Simulation", "config", "parse_input", "load_library", "lib_path", "FIELDS",
           "MODELS", "DBA_ERR", "OPT_WAIT_LIMIT", "BATCH_PERSISTENT", "BATCH_WAIT_LIMIT"]
