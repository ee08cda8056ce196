"""Host-side world container of the XPBD creature step (src/physics/xpbd.js).

``XpbdWorld`` holds exactly the state the reference's XpbdWorld holds
(xpbd.js:188-247): flat float64 body arrays grown by doubling, collision
sample points and the constraint list in solve order.  It has no CPU physics
step -- the step runs on the GPU through :mod:`kraken_3_gpu_b200.gpuworld`.

Colouring (assignColor / ensureColored, xpbd.js:98-126) lives here as in the
reference, because gpuworld.create calls it defensively.
"""
from __future__ import annotations

import math

import numpy as np

# xpbd.js:46-54
SOLVER_DEFAULTS = {
    "substeps": 2,
    "iterations": 4,
    "h": 1 / 120,
    "linDrag": 3.0,
    "angDrag": 3.0,
    "maxSpeed": 360,
    "maxAngSpeed": 18,
}

SLACK_POS = 2e-3  # xpbd.js:77
SLACK_ANG = 2e-4  # xpbd.js:78
MAX_COLORS = 16   # xpbd.js:96

C_PIN = 0    # xpbd.js:148
C_ANGLE = 1  # xpbd.js:149
C_GRIP = 2   # xpbd.js:150

_ARRAYS = ("px", "py", "ppx", "ppy", "vx", "vy", "ang", "angP", "av", "im", "ii",
           "fx", "fy", "tq")


def assign_color(color_mask, a: int, b: int) -> int:
    """assignColor, xpbd.js:98-105: smallest colour free at both bodies.

    ``color_mask`` behaves like the reference's Uint32Array: a read past its
    end gives 0 and a write past its end is dropped (createSim allocates
    1 << 16 entries, core.js:45, so bodies beyond that always see colour 0
    free).  Only the colour labels change; the solve order stays the list
    order the colours produce, which the GPU schedule reproduces exactly."""
    n = len(color_mask)
    ma = int(color_mask[a]) if a < n else 0
    mb = (int(color_mask[b]) if b < n else 0) if b >= 0 else 0
    used = ma | mb
    c = 0
    while used & (1 << c):
        c += 1
    if a < n:
        color_mask[a] = ma | (1 << c)
    if 0 <= b < n:
        color_mask[b] = mb | (1 << c)
    return c


def wrap_angle(a: float) -> float:
    """wrapAngle, xpbd.js:128-134 (JS `%` is fmod)."""
    tau = math.pi * 2
    d = math.fmod(a, tau)
    if d > math.pi:
        d -= tau
    elif d < -math.pi:
        d += tau
    return d


def angle_delta(a: float, b: float) -> float:
    """angleDelta, xpbd.js:137-143."""
    try:
        d = math.fmod(a - b, math.pi * 2)
    except ValueError:
        return 0.0
    if not math.isfinite(d):
        return 0.0
    if d > math.pi:
        d -= math.pi * 2
    elif d < -math.pi:
        d += math.pi * 2
    return d


class Constraint:
    """makeConstraint, xpbd.js:160-179 -- every field the reference carries."""

    __slots__ = ("type", "a", "b", "lax", "lay", "lbx", "lby", "compliance", "lambda_",
                 "lambdaX", "lambdaY", "broken", "breakForce", "force", "target", "rest",
                 "minAngle", "maxAngle", "owner", "color")

    def __init__(self, type_, a, b, lax, lay, lbx, lby, compliance=0.0):
        self.type = type_
        self.a = a
        self.b = b
        self.lax = lax
        self.lay = lay
        self.lbx = lbx
        self.lby = lby
        self.compliance = compliance
        self.lambda_ = 0.0
        self.lambdaX = 0.0
        self.lambdaY = 0.0
        self.broken = False
        self.breakForce = math.inf
        self.force = 0.0
        self.target = 0.0
        self.rest = 0.0
        self.minAngle = -math.inf
        self.maxAngle = math.inf
        self.owner = -1
        self.color = -1

    # `lambda` is a Python keyword; keep the reference's name reachable
    @property
    def lam(self):
        return self.lambda_

    @lam.setter
    def lam(self, v):
        self.lambda_ = v


def make_constraint(type_, a, b, lax, lay, lbx, lby, compliance=0.0) -> Constraint:
    return Constraint(type_, a, b, lax, lay, lbx, lby, compliance)


class CollPt:
    __slots__ = ("body", "lx", "ly", "r")

    def __init__(self, body, lx, ly, r):
        self.body, self.lx, self.ly, self.r = body, lx, ly, r


class XpbdWorld:
    """State of the reference's XpbdWorld without its CPU step (xpbd.js:188-247)."""

    def __init__(self, **opts):
        o = {**SOLVER_DEFAULTS, **opts}
        self.substeps = o["substeps"]
        self.iterations = o["iterations"]
        self.h = o["h"]
        self.linDrag = o["linDrag"]
        self.angDrag = o["angDrag"]
        self.maxSpeed = o["maxSpeed"]
        self.maxAngSpeed = o["maxAngSpeed"]
        self.n = 0
        self.cap = 0
        for name in _ARRAYS:
            setattr(self, name, None)
        self.collPts: list[CollPt] = []
        self.constraints: list[Constraint] = []
        self.sdf = None
        self.stats = {"maxSpeed": 0.0, "maxAngSpeed": 0.0, "nan": 0, "collisions": 0, "broken": 0}
        self.colorOff = None
        self.colorCnt = None
        self.colorMax = 0

    def add_body(self, x, y, angle, mass, inertia) -> int:
        """addBody, xpbd.js:217-228."""
        i = self.n
        self.n += 1
        if i >= self.cap:
            self._grow()
        self.px[i] = x
        self.py[i] = y
        self.ppx[i] = x
        self.ppy[i] = y
        self.vx[i] = 0
        self.vy[i] = 0
        self.ang[i] = angle
        self.angP[i] = angle
        self.av[i] = 0
        self.im[i] = 1 / mass if mass > 0 else 0
        self.ii[i] = 1 / inertia if inertia > 0 else 0
        self.fx[i] = 0
        self.fy[i] = 0
        self.tq[i] = 0
        return i

    addBody = add_body

    def _grow(self):
        """_grow, xpbd.js:230-240."""
        cap = max(64, self.cap * 2)
        for name in _ARRAYS:
            d = np.zeros(cap, dtype=np.float64)
            src = getattr(self, name)
            if src is not None:
                d[: len(src)] = src
            setattr(self, name, d)
        self.cap = cap

    def add_collision_point(self, body, lx, ly, r):
        """addCollisionPoint, xpbd.js:243-245."""
        self.collPts.append(CollPt(body, lx, ly, r))

    addCollisionPoint = add_collision_point

    def add_constraint(self, c: Constraint) -> Constraint:
        self.constraints.append(c)
        return c

    addConstraint = add_constraint

    def step(self):
        raise NotImplementedError(
            "XpbdWorld has no CPU step here; advance it on the GPU with gpuworld.step()")


def ensure_colored(world: XpbdWorld):
    """ensureColored, xpbd.js:108-126: colour uncoloured constraints in list
    order with a fresh mask, then group the list stably by colour."""
    if world.colorOff is not None:
        return world.colorOff
    mask = np.zeros(max(1024, world.n * 2), dtype=np.uint32)
    for c in world.constraints:
        if c.color < 0:
            c.color = assign_color(mask, c.a, c.b if c.b >= 0 else -1)
    _group(world)
    return world.colorOff


def _group(world: XpbdWorld):
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
