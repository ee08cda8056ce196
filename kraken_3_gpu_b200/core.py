"""Simulation core around the physics step (src/sim/core.js): world
construction with the constraint colouring, the control write-back with the
suction-cup slip-gate reflex, and the 42-value proprioception vector.

Senses, prey, lights and fitness bookkeeping of core.js are not on the
physics path and are not reproduced; ``create_sim`` builds the same world,
map and creatures in the same random order as createSim with ``prey: 0``.
"""
from __future__ import annotations

import math

import numpy as np

from .kraken import (BODY, arm_curl, arm_extension, arm_reach, attach_grip,
                     adhesion_to_break_force, release_grip, spawn_kraken, tip_position,
                     tone_to_compliance)
from .world_map import find_spawn, make_map, mulberry32
from .xpbd import MAX_COLORS, XpbdWorld, assign_color

# core.js:19-35 (physics-relevant entries)
DEFAULTS = {
    "width": 1440, "height": 810, "seed": 1, "creatures": 1, "substeps": 2,
    "iterations": 4, "h": 1 / 120, "gripSlipMax": 150, "gripCooldown": 0.05,
    "arms": BODY["arms"], "segsPerArm": BODY["segsPerArm"],
}

PROPRIO_DIM = 42  # core.js:123 (6 per arm + 6, for six arms)


def proprio_dim(arms: int) -> int:
    return 6 * arms + 6


class Creature:
    """makeCreature, core.js:76-97 (control and proprioception state)."""

    def __init__(self, world, k, opts, index):
        self.index = index
        self.mantle = k.mantle
        self.arms = k.arms
        self.spawn = k.spawn
        self.opts = opts
        self.world = world
        self.tone = 0.5
        self.perArm = [{"shoulder": 0.0, "curl": 0.0, "adhesion": 0.0, "cd": 0.0} for _ in k.arms]
        self.prevVx = 0.0
        self.prevVy = 0.0
        self.x = self.y = self.vx = self.vy = self.angle = self.av = self.speed = 0.0
        self.anchoredCount = 0
        self.meanExtension = 1.0
        self.meanCurl = 0.0
        self.reach = arm_reach(len(k.arms[0].segs)) if k.arms else arm_reach()


def group_constraints_by_color(world: XpbdWorld):
    """groupConstraintsByColor, core.js:276-288."""
    buckets = [[] for _ in range(MAX_COLORS)]
    for c in world.constraints:
        buckets[c.color | 0].append(c)
    off = np.zeros(MAX_COLORS, dtype=np.uint32)
    cnt = np.zeros(MAX_COLORS, dtype=np.uint32)
    n = 0
    max_cnt = 0
    for c in range(MAX_COLORS):
        off[c] = n
        cnt[c] = len(buckets[c])
        max_cnt = max(max_cnt, len(buckets[c]))
        n += len(buckets[c])
    world.constraints = [c for b in buckets for c in b]
    world.colorOff = off
    world.colorCnt = cnt
    world.colorMax = max_cnt


def create_sim(**opts):
    """createSim, core.js:37-74 with prey 0 and an optional body shape.
    poses: optional (x, y, angle) per creature instead of findSpawn's points
    and the seeded headings (the map is still makeMap of the seed)."""
    o = {**DEFAULTS, **opts}
    poses = o.pop("poses", None)
    if poses is not None:
        o["creatures"] = len(poses)
    world = XpbdWorld(substeps=o["substeps"], iterations=o["iterations"], h=o["h"])
    m = make_map(o["width"], o["height"], seed=o["seed"])
    world.sdf = m["sdf"]
    rnd = mulberry32((o["seed"] ^ 0x9E3779B9) & 0xFFFFFFFF)
    creatures = []
    color_mask = np.zeros(1 << 16, dtype=np.uint32)
    colored_upto = 0
    for i in range(o["creatures"]):
        if poses is not None:
            x, y, ang = (float(v) for v in poses[i])
        else:
            sp = find_spawn(m, arm_reach(o["segsPerArm"]) + 20, rnd)
            x, y, ang = sp["x"], sp["y"], rnd() * math.pi * 2
        k = spawn_kraken(world, x, y, ang, arms=o["arms"], segs=o["segsPerArm"])
        # core.js:51-58: colour this creature's constraints (global body mask)
        for c in world.constraints[colored_upto:]:
            if c.color < 0:
                c.color = assign_color(color_mask, c.a, c.b if c.b >= 0 else -1)
        colored_upto = len(world.constraints)
        creatures.append(Creature(world, k, o, i))
    group_constraints_by_color(world)
    return {"world": world, "map": m, "creatures": creatures, "entities": [], "opts": o,
            "rnd": rnd, "time": 0, "stepCount": 0}


def read_state(c: Creature):
    """readState, core.js:100-107."""
    w, m = c.world, c.mantle
    c.x, c.y = w.px[m], w.py[m]
    c.vx, c.vy = w.vx[m], w.vy[m]
    c.angle, c.av = w.ang[m], w.av[m]
    c.speed = math.hypot(c.vx, c.vy)
    return c


def _reflex(c: Creature, a: int, adhesion: float):
    """Suction-cup reflex of applyControl, core.js:199-218."""
    w = c.world
    arm, st = c.arms[a], c.perArm[a]
    st["adhesion"] = max(0, min(1, adhesion))
    if st["cd"] > 0:
        st["cd"] -= w.h * w.substeps
    g = arm.grip
    if g.broken:
        if st["adhesion"] > 0.08 and st["cd"] <= 0:
            slip = math.hypot(w.vx[arm.tip], w.vy[arm.tip])
            if slip < c.opts["gripSlipMax"]:
                attach_grip(w, arm, adhesion_to_break_force(st["adhesion"]))
            else:
                st["cd"] = c.opts["gripCooldown"]
    else:
        g.breakForce = adhesion_to_break_force(st["adhesion"])
        if st["adhesion"] < 0.04:
            release_grip(arm)


def apply_control(c: Creature, control: dict):
    """applyControl, core.js:183-220 (tone, per-arm shoulder/curl/adhesion)."""
    c.tone = max(0, min(1, control["tone"]))
    comp = tone_to_compliance(c.tone)
    for a, arm in enumerate(c.arms):
        ctl = control["arms"][a]
        for m in arm.motors:
            m.compliance = comp
        arm.motors[0].target = max(-BODY["shoulderLimit"], min(BODY["shoulderLimit"], ctl["shoulder"]))
        for j in range(1, len(arm.motors)):
            arm.motors[j].target = max(-BODY["jointLimit"], min(BODY["jointLimit"], ctl["curl"]))
        _reflex(c, a, ctl["adhesion"])


def apply_control_motors(c: Creature, tone: float, targets, adhesion):
    """applyControl with one commanded deviation per motor (arm-major,
    motor 0 = shoulder), clamped exactly as core.js:195-198 clamps."""
    c.tone = max(0, min(1, tone))
    comp = tone_to_compliance(c.tone)
    k = 0
    for a, arm in enumerate(c.arms):
        for j, m in enumerate(arm.motors):
            m.compliance = comp
            lim = BODY["shoulderLimit"] if j == 0 else BODY["jointLimit"]
            m.target = max(-lim, min(lim, float(targets[k])))
            k += 1
        _reflex(c, a, float(adhesion[a]))


def read_proprio(c: Creature, out=None):
    """readProprio, core.js:129-175: 6 values per arm + 6 body values."""
    w = c.world
    read_state(c)
    A = len(c.arms)
    if out is None:
        out = np.zeros(6 * A + 6)
    ca, sa = math.cos(-c.angle), math.sin(-c.angle)
    anchored, ext_sum, curl_sum = 0, 0.0, 0.0
    shoulder = []
    for arm in c.arms:
        d = w.ang[arm.segs[0]] - c.angle
        shoulder.append(math.atan2(math.sin(d), math.cos(d)))
        ext_sum += arm_extension(w, arm, c.reach)
        curl_sum += arm_curl(w, arm)
        if not arm.grip.broken:
            anchored += 1

    def cl(v, m):
        return m if v > m else (-m if v < -m else v)

    i = 0
    for a in range(A):
        out[i] = cl(shoulder[a] / BODY["shoulderLimit"], 1.2); i += 1
    for a in range(A):
        out[i] = cl(arm_curl(w, c.arms[a]) / BODY["jointLimit"], 1.2); i += 1
    for a in range(A):
        t = tip_position(w, c.arms[a])
        dx, dy = t["x"] - c.x, t["y"] - c.y
        out[i] = cl((dx * ca - dy * sa) / c.reach, 1.2); i += 1
        out[i] = cl((dx * sa + dy * ca) / c.reach, 1.2); i += 1
    for a in range(A):
        g = c.arms[a].grip
        f = g.force if g.force == g.force else 0.0
        out[i] = 0 if g.broken else min(1, (f or 0) / max(1, g.breakForce)); i += 1
    for a in range(A):
        out[i] = 0 if c.arms[a].grip.broken else 1; i += 1
    ax = (c.vx - c.prevVx) / (w.h * w.substeps)
    ay = (c.vy - c.prevVy) / (w.h * w.substeps)
    out[i] = max(-1, min(1, (ax * ca - ay * sa) / 600)); i += 1
    out[i] = max(-1, min(1, (ax * sa + ay * ca) / 600)); i += 1
    c.prevVx, c.prevVy = c.vx, c.vy
    out[i] = anchored / A; i += 1
    c.meanExtension = ext_sum / A
    c.meanCurl = curl_sum / A
    out[i] = c.meanExtension; i += 1
    out[i] = min(1, c.speed / 300); i += 1
    out[i] = max(-1, min(1, c.av / 18)); i += 1
    c.anchoredCount = anchored
    return out


createSim = create_sim
readState = read_state
applyControl = apply_control
readProprio = read_proprio
groupConstraintsByColor = group_constraints_by_color
