"""cgfdm: B200-native (sm_100a) time-stepping hot path of CGFDM.

The compute path is the CUDA library lib/libcgfdm_b200.so behind the C ABI of
include/cgfdm_b200.h; this package is its Python host binding.
"""
from ._lib import (BF16, FP16, FP32, FP64, KERNEL_AUTO, KERNEL_EXACT, KERNEL_STREAM, LIB_PATH,
                   REQ_CANCELLED, REQ_DONE, REQ_FAILED, REQ_QUEUED, REQ_RUNNING, CgfdmError, lib)
from .api import (Batch, Server, Simulation, device_bytes, hbm_layout, make_desc, propagate, run_directory,
                  setup_from_directory, stage_noalloc)

__all__ = ["Simulation", "Batch", "Server", "propagate", "setup_from_directory", "run_directory", "make_desc",
           "device_bytes", "CgfdmError", "lib", "LIB_PATH", "FP32", "FP16", "BF16", "FP64",
           "KERNEL_AUTO", "KERNEL_EXACT", "KERNEL_STREAM", "hbm_layout", "stage_noalloc"]
