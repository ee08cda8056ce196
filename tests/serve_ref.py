"""Host restatement of the server's eps generator (splitmix64 of (seed, pair,
parameter) -> two 24-bit uniforms -> Box-Muller) and of the mirrored weights
theta +- sigma * eps, used to check the device."""
import numpy as np

M64 = (1 << 64) - 1


def splitmix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def eps(seed: int, pair: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float64)
    for p in range(n):
        x = splitmix64((seed & M64) ^ splitmix64(((pair & 0xFFFFFFFF) << 32) | p))
        u1 = ((x >> 40) + 1.0) / 16777216.0
        u2 = (x & 0xFFFFFF) / 16777216.0
        out[p] = np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
    return out


def mirrored_weights(theta, sigma, eps_k, sign):
    """f32(theta + f32(+-f32(sigma * eps))), as the device rounds it."""
    d = np.float32(sigma) * eps_k.astype(np.float32)
    return (theta.astype(np.float32) + (d if sign > 0 else -d)).astype(np.float32)
