"""Body model: mantle + arms of segments, one suction cup per arm
(src/body/kraken.js), with the arm and segment count as parameters.

The reference hard-codes BODY.arms = 6 and BODY.segsPerArm = 7
(kraken.js:23-24); ``spawn_kraken`` takes both as arguments and keeps every
other constant and the construction order, so the default body is the
reference's body bit for bit.
"""
from __future__ import annotations

import math

from .xpbd import C_ANGLE, C_GRIP, C_PIN, XpbdWorld, make_constraint

# kraken.js:22-47
BODY = {
    "arms": 6,
    "segsPerArm": 7,
    "segLen": 13.5,
    "shoulderR": 24,
    "mantleRadius": 18,
    "mantleMass": 20,
    "mantleInertiaFactor": 2.5,
    "segMassProx": 3.2,
    "segMassDist": 1.8,
    "segThickProx": 11.9,
    "segThickDist": 5.9,
    "jointLimit": math.pi * 0.42,
    "shoulderLimit": math.pi * 0.62,
    "spawnCurl": 0.28,
    "muscleStiffnessMin": 2000,
    "muscleStiffnessMax": 400000,
    "gripBreakMin": 40,
    "gripBreakMax": 900,
}


def arm_reach(segs: int = BODY["segsPerArm"]) -> float:
    """ARM_REACH, kraken.js:49, for a given segment count."""
    return BODY["shoulderR"] + segs * BODY["segLen"]


ARM_REACH = arm_reach()


def _rect_inertia(m, w, h):
    return m * (w * w + h * h) / 12


class Arm:
    __slots__ = ("relAng", "segs", "motors", "grip", "tip", "index")

    def __init__(self, relAng, segs, motors, grip, tip, index):
        self.relAng, self.segs, self.motors = relAng, segs, motors
        self.grip, self.tip, self.index = grip, tip, index


class Kraken:
    __slots__ = ("mantle", "arms", "spawn")

    def __init__(self, mantle, arms, spawn):
        self.mantle, self.arms, self.spawn = mantle, arms, spawn


def spawn_kraken(world: XpbdWorld, x, y, angle, curl=None, arms=None, segs=None) -> Kraken:
    """spawnKraken, kraken.js:64-148 (constraint-free pose, then constraints)."""
    B = BODY
    curl = B["spawnCurl"] if curl is None else curl
    n_arms = B["arms"] if arms is None else int(arms)
    n_segs = B["segsPerArm"] if segs is None else int(segs)
    mantle_i = (B["mantleMass"] * B["mantleRadius"] * B["mantleRadius"] / 2) * B["mantleInertiaFactor"]
    mantle = world.add_body(x, y, angle, B["mantleMass"], mantle_i)
    for i in range(8):
        a = (i / 8) * math.pi * 2
        world.add_collision_point(mantle, math.cos(a) * B["mantleRadius"] * 0.7,
                                  math.sin(a) * B["mantleRadius"] * 0.7, B["mantleRadius"] * 0.45)
    out = []
    for a in range(n_arms):
        rel_ang = (a / n_arms) * math.pi * 2
        th0 = angle + rel_ang
        segs_l = []
        jx = x + math.cos(th0) * B["shoulderR"]
        jy = y + math.sin(th0) * B["shoulderR"]
        th = th0
        for i in range(n_segs):
            t = i / (n_segs - 1) if n_segs > 1 else 0
            mass = B["segMassProx"] + (B["segMassDist"] - B["segMassProx"]) * t
            thick = B["segThickProx"] + (B["segThickDist"] - B["segThickProx"]) * t
            ux, uy = math.cos(th), math.sin(th)
            cx = jx + ux * B["segLen"] * 0.5
            cy = jy + uy * B["segLen"] * 0.5
            b = world.add_body(cx, cy, th, mass, _rect_inertia(mass, B["segLen"], thick))
            r = thick * 0.5
            world.add_collision_point(b, -B["segLen"] * 0.5 + r * 0.4, 0, r)
            world.add_collision_point(b, B["segLen"] * 0.5 - r * 0.4, 0, r)
            segs_l.append(b)
            jx = cx + ux * B["segLen"] * 0.5
            jy = cy + uy * B["segLen"] * 0.5
            th += curl
        world.add_constraint(make_constraint(C_PIN, mantle, segs_l[0],
                                             math.cos(rel_ang) * B["shoulderR"],
                                             math.sin(rel_ang) * B["shoulderR"],
                                             -B["segLen"] * 0.5, 0, 0))
        motors = []
        m_sh = make_constraint(C_ANGLE, mantle, segs_l[0], 0, 0, 0, 0, 1 / B["muscleStiffnessMin"])
        m_sh.rest = rel_ang
        m_sh.target = 0
        m_sh.minAngle = -B["shoulderLimit"]
        m_sh.maxAngle = B["shoulderLimit"]
        m_sh.owner = a
        world.add_constraint(m_sh)
        motors.append(m_sh)
        for i in range(len(segs_l) - 1):
            world.add_constraint(make_constraint(C_PIN, segs_l[i], segs_l[i + 1],
                                                 B["segLen"] * 0.5, 0, -B["segLen"] * 0.5, 0, 0))
            motor = make_constraint(C_ANGLE, segs_l[i], segs_l[i + 1], 0, 0, 0, 0,
                                    1 / B["muscleStiffnessMin"])
            motor.rest = curl
            motor.target = 0
            motor.minAngle = -B["jointLimit"]
            motor.maxAngle = B["jointLimit"]
            motor.owner = a
            world.add_constraint(motor)
            motors.append(motor)
        tip = segs_l[-1]
        grip = make_constraint(C_GRIP, tip, -1, B["segLen"] * 0.5, 0, x, y, 0)
        grip.broken = True
        grip.breakForce = 0
        grip.owner = a
        world.add_constraint(grip)
        out.append(Arm(rel_ang, segs_l, motors, grip, tip, a))
    return Kraken(mantle, out, {"x": x, "y": y, "angle": angle})


def tip_position(world: XpbdWorld, arm: Arm):
    """tipPosition, kraken.js:150-154."""
    b = arm.tip
    L = BODY["segLen"] * 0.5
    c, s = math.cos(world.ang[b]), math.sin(world.ang[b])
    return {"x": world.px[b] + L * c, "y": world.py[b] + L * s}


def attach_grip(world: XpbdWorld, arm: Arm, break_force):
    """attachGrip, kraken.js:157-164."""
    t = tip_position(world, arm)
    g = arm.grip
    g.lbx, g.lby = t["x"], t["y"]
    g.broken = False
    g.breakForce = break_force
    g.lambdaX = 0
    g.lambdaY = 0
    g.force = 0
    return g


def release_grip(arm: Arm):
    """releaseGrip, kraken.js:166."""
    arm.grip.broken = True
    arm.grip.force = 0


def arm_curl(world: XpbdWorld, arm: Arm) -> float:
    """armCurl, kraken.js:169-176."""
    s, n = 0.0, 0
    for i in range(1, len(arm.segs)):
        d = world.ang[arm.segs[i]] - world.ang[arm.segs[i - 1]]
        s += math.atan2(math.sin(d), math.cos(d))
        n += 1
    return s / n if n else 0.0


def arm_extension(world: XpbdWorld, arm: Arm, reach: float = ARM_REACH) -> float:
    """armExtension, kraken.js:179-183."""
    t = tip_position(world, arm)
    s0 = arm.segs[0]
    return min(1, math.hypot(t["x"] - world.px[s0], t["y"] - world.py[s0]) / max(1, reach))


def tone_to_compliance(tone: float) -> float:
    """toneToCompliance, kraken.js:186-191."""
    B = BODY
    t = max(0, min(1, tone))
    stiff = B["muscleStiffnessMin"] + t * (B["muscleStiffnessMax"] - B["muscleStiffnessMin"])
    return 1 / stiff


def adhesion_to_break_force(a: float) -> float:
    """adhesionToBreakForce, kraken.js:194-198."""
    B = BODY
    c = max(0, min(1, a))
    return B["gripBreakMin"] + (B["gripBreakMax"] - B["gripBreakMin"]) * c


spawnKraken = spawn_kraken
tipPosition = tip_position
attachGrip = attach_grip
releaseGrip = release_grip
armCurl = arm_curl
armExtension = arm_extension
toneToCompliance = tone_to_compliance
adhesionToBreakForce = adhesion_to_break_force
