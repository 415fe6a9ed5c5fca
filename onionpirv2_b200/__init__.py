"""B200-native (sm_100a) OnionPIRv2 server hot path.

The compute lives in libonionpir_b200.so (CUDA kernels behind a C ABI, see
include/onionpir_b200.h); this package is the host-side mirror of the
reference's PirParams / PirServer interface over that ABI, plus the
client's batchable steps (PirClient: query packing and decryption).
"""
from .server import (DeviceError, OutOfRange, PirParams, PirServer,  # noqa: F401
                     RowShardServer, plan_memory, row_shard_rows, save_response)
from .client import PirClient  # noqa: F401,E402

__all__ = ["PirParams", "PirServer", "PirClient", "RowShardServer", "row_shard_rows",
           "save_response", "plan_memory", "OutOfRange", "DeviceError"]
