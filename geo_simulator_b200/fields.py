"""Seeded synthetic inputs of the benchmark configurations (host, FP64).

Every random field is generated once on the host, so the GPU path and the CPU
oracle see identical bits: splitmix64(seed, index) gives two uniforms in (0, 1]
per entry, Box-Muller turns them into a standard normal.
"""
from __future__ import annotations

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, counter: np.ndarray) -> np.ndarray:
    """splitmix64 output for state seed + (counter + 1) * golden, vectorised (uint64)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (counter.astype(np.uint64) + np.uint64(1)) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, counter: np.ndarray) -> np.ndarray:
    """Uniforms in (0, 1] with 53 random bits."""
    z = splitmix64(seed, counter)
    return ((z >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int) -> np.ndarray:
    i = np.arange(n, dtype=np.uint64)
    u1 = uniform01(seed, np.uint64(2) * i)
    u2 = uniform01(seed, np.uint64(2) * i + np.uint64(1))
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)


def lognormal_field(seed: int, n: int, mean_log: float, sigma_log: float, log: bool = False) -> np.ndarray:
    """exp(mean_log + sigma_log * N(0, 1)) per entry (or the log itself when log=True)."""
    v = mean_log + sigma_log * normal(seed, n)
    return v if log else np.exp(v)


def choice_distinct(seed: int, n_pool: int, k: int) -> np.ndarray:
    """k distinct indices of range(n_pool), seeded (sorted uniforms of the pool)."""
    keys = splitmix64(seed, np.arange(n_pool, dtype=np.uint64))
    return np.sort(np.argsort(keys, kind="stable")[:k])
