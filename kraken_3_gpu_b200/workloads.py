"""Seeded synthetic workloads of the batched engine.

uneven(n=16384, maps=64): creatures of 4-8 arms x 5-9 segments on maps whose
  corridor-grid density is drawn from U[0.1, 0.4] per map, horizons from
  U{200..2000}; every draw from mulberry32 streams (src/world/map.js:11-20).
uniform(n=1024): default bodies on map seed 1, spawned around the
  findSpawn point of the map with jitter U[-20, 20] px and heading U[0, 2 pi).

Spawn points follow findSpawn (map.js:120-128) with the body's arm reach + 20
px clearance, as createSim does (core.js:49).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .kraken import arm_reach
from .world_map import find_spawn, light_array, make_map, mulberry32

WIDTH, HEIGHT = 1440, 810
TONE = 0.5  # creature default tone, core.js:81 (compliance 1 / 201000)


class ControlStream:
    """Host mirror of the engine's device control stream: per arm-segment
    muscle targets ~ U[-1, 1] rad and per-arm adhesion ~ U[0, 1], redrawn
    every `every` env steps from mulberry32(seed); draw order per arm: its
    motors (shoulder first), then its adhesion."""

    def __init__(self, n_arms=6, n_segs=7, seed=0, every=6):
        self.rnd = mulberry32(seed)
        self.A, self.S, self.every = n_arms, n_segs, every
        self.targets = np.zeros(n_arms * n_segs)
        self.adhesion = np.zeros(n_arms)

    def at(self, step):
        if step % self.every == 0:
            for a in range(self.A):
                for j in range(self.S):
                    self.targets[a * self.S + j] = self.rnd() * 2 - 1
                self.adhesion[a] = self.rnd()
        return self.targets, self.adhesion


@dataclass
class Workload:
    name: str
    maps: list            # list of (n, 4) float arrays x y w h
    arms: np.ndarray
    segs: np.ndarray
    map_id: np.ndarray
    x: np.ndarray
    y: np.ndarray
    angle: np.ndarray
    horizon: np.ndarray
    seed: np.ndarray      # control stream seed per creature
    lights: list = None   # per map (n, 6) f64: x y r ir ph sp (makeMap's moving lights)

    @property
    def n(self) -> int:
        return len(self.x)

    def creature_steps(self) -> int:
        return int(self.horizon.sum())


def _rects(m):
    return np.array([[r["x"], r["y"], r["w"], r["h"]] for r in m["rects"]], dtype=np.float64)


def uneven(n=16384, n_maps=64, seed=2, h_min=200, h_max=2000, arms=(4, 8), segs=(5, 9)) -> Workload:
    rnd = mulberry32(seed)
    maps_js = []
    for m in range(n_maps):
        density = 0.1 + 0.3 * rnd()
        maps_js.append(make_map(WIDTH, HEIGHT, seed=1000 * seed + m, density=density))
    A = np.zeros(n, np.int32); S = np.zeros(n, np.int32); M = np.zeros(n, np.int32)
    X = np.zeros(n); Y = np.zeros(n); ANG = np.zeros(n); H = np.zeros(n, np.int32)
    spawn_rng = [mulberry32((seed * 7919 + m) ^ 0x9E3779B9) for m in range(n_maps)]
    for i in range(n):
        A[i] = arms[0] + math.floor(rnd() * (arms[1] - arms[0] + 1))
        S[i] = segs[0] + math.floor(rnd() * (segs[1] - segs[0] + 1))
        M[i] = math.floor(rnd() * n_maps)
        H[i] = h_min + math.floor(rnd() * (h_max - h_min + 1))
        r = spawn_rng[M[i]]
        sp = find_spawn(maps_js[M[i]], arm_reach(int(S[i])) + 20, r)
        X[i], Y[i] = sp["x"], sp["y"]
        ANG[i] = r() * math.pi * 2
    seeds = (np.arange(n, dtype=np.uint64) * 2654435761 + seed).astype(np.uint32)
    return Workload("uneven", [_rects(m) for m in maps_js], A, S, M, X, Y, ANG, H, seeds,
                    [np.array(light_array(m), dtype=np.float64).reshape(-1, 6) for m in maps_js])


def uniform(n=1024, steps=1000, map_seed=1, seed=1, jitter=20.0) -> Workload:
    m = make_map(WIDTH, HEIGHT, seed=map_seed)
    base = find_spawn(m, arm_reach() + 20, mulberry32((map_seed ^ 0x9E3779B9) & 0xFFFFFFFF))
    rnd = mulberry32(seed)
    X = np.zeros(n); Y = np.zeros(n); ANG = np.zeros(n)
    for i in range(n):
        X[i] = base["x"] + (rnd() * 2 - 1) * jitter
        Y[i] = base["y"] + (rnd() * 2 - 1) * jitter
        ANG[i] = rnd() * math.pi * 2
    ones = np.ones(n, np.int32)
    seeds = (np.arange(n, dtype=np.uint64) * 2654435761 + seed).astype(np.uint32)
    return Workload("uniform", [_rects(m)], 6 * ones, 7 * ones, 0 * ones, X, Y, ANG,
                    steps * ones, seeds, [np.array(light_array(m), dtype=np.float64).reshape(-1, 6)])


def spawn_all(engine, w: Workload, first=0):
    engine.spawn(first, w.arms, w.segs, w.map_id, w.x, w.y, w.angle, w.horizon, w.seed)
