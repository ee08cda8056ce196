"""Seeded scenarios shared by the GPU tests.

ControlStream (from the package): per arm-segment muscle targets ~ U[-1, 1]
rad and per-arm adhesion ~ U[0, 1], redrawn every 6 env steps from
mulberry32(seed), draw order per arm: its motors (shoulder first), then its
adhesion.  Tone is fixed at 0.5 (compliance 1/201000, the creature default of
core.js:81).
"""
import numpy as np

from kraken_3_gpu_b200.workloads import TONE, ControlStream  # noqa: F401


def ulp_distance(a32: np.ndarray, b32: np.ndarray) -> np.ndarray:
    """ulp distance between two float32 arrays (ordered integer mapping)."""
    ai = np.asarray(a32, dtype=np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b32, dtype=np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, np.int64(-0x80000000) - ai, ai)
    bi = np.where(bi < 0, np.int64(-0x80000000) - bi, bi)
    return np.abs(ai - bi)
