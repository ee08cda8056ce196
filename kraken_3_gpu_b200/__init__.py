"""kraken_3_gpu_b200 -- Kraken 3's XPBD creature step on NVIDIA B200 (sm_100a).

Layers:
  csrc/ + libkraken_b200.so   CUDA kernels and the C ABI (include/kraken_b200.h)
  gpuworld                    drop-in of src/gpu/gpuworld.js over that ABI
  xpbd, world_map, kraken,    host-side world builders of src/physics/xpbd.js,
  core                        src/world/map.js, src/body/kraken.js, src/sim/core.js
"""
from . import core, gpuworld, kraken, world_map, xpbd  # noqa: F401

__all__ = ["core", "gpuworld", "kraken", "world_map", "xpbd"]
