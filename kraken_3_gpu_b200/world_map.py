"""Map as a rect list plus the analytic SDF (src/world/map.js).

Host-side: map generation runs once per map; the SDF here serves spawn
placement.  The per-substep SDF of the collision pass runs in the CUDA
kernel over the same rect list.
"""
from __future__ import annotations

import math


def mulberry32(seed: int):
    """mulberry32, map.js:11-20 (uint32 arithmetic, as JS >>> 0 / Math.imul)."""
    state = [seed & 0xFFFFFFFF]

    def rnd() -> float:
        a = (state[0] + 0x6D2B79F5) & 0xFFFFFFFF
        state[0] = a
        t = a
        t = ((t ^ (t >> 15)) * (t | 1)) & 0xFFFFFFFF
        t ^= (t + (((t ^ (t >> 7)) * (t | 61)) & 0xFFFFFFFF)) & 0xFFFFFFFF
        return ((t ^ (t >> 14)) & 0xFFFFFFFF) / 4294967296

    return rnd


def make_map(width, height, **opts):
    """makeMap, map.js:22-71: rects, the SDF and the moving lights (drawn
    after the rects from the same stream; only the light sense reads them)."""
    o = {"wallThickness": 14, "corridorCols": 4, "corridorRows": 3, "density": 0.48,
         "seed": 1, **opts}
    rects = []
    T = o["wallThickness"]
    rects.append({"x": 0, "y": 0, "w": width, "h": T})
    rects.append({"x": 0, "y": height - T, "w": width, "h": T})
    rects.append({"x": 0, "y": 0, "w": T, "h": height})
    rects.append({"x": width - T, "y": 0, "w": T, "h": height})
    rnd = mulberry32(o["seed"])
    cols, rows, density = o["corridorCols"], o["corridorRows"], o["density"]
    cw, ch = width / cols, height / rows
    for col in range(1, cols):
        xl = col * cw
        for row in range(rows):
            if rnd() > density:
                continue
            ys = row * ch
            g_sz = max(60, min(ch * (0.28 + rnd() * 0.38), height * 0.4))
            g_start = ys + rnd() * max(1, ch - g_sz)
            wt = 10 + math.floor(rnd() * 10)
            if g_start > ys + 14:
                rects.append({"x": xl - wt / 2, "y": ys, "w": wt, "h": g_start - ys})
            g_end = g_start + g_sz
            if g_end < ys + ch - 14:
                rects.append({"x": xl - wt / 2, "y": g_end, "w": wt, "h": ys + ch - g_end})
    for row in range(1, rows):
        yl = row * ch
        for col in range(cols):
            if rnd() > density:
                continue
            xs = col * cw
            g_sz = max(60, min(cw * (0.28 + rnd() * 0.38), width * 0.3))
            g_start = xs + rnd() * max(1, cw - g_sz)
            wt = 10 + math.floor(rnd() * 10)
            if g_start > xs + 14:
                rects.append({"x": xs, "y": yl - wt / 2, "w": g_start - xs, "h": wt})
            g_end = g_start + g_sz
            if g_end < xs + cw - 14:
                rects.append({"x": g_end, "y": yl - wt / 2, "w": xs + cw - g_end, "h": wt})
    lights = []
    for _ in range(o.get("lights", 4)):
        x = T + rnd() * max(1, width - T * 2)      # findSpawnRaw, map.js:72-74
        y = T + rnd() * max(1, height - T * 2)
        r = 220 + rnd() * 70
        ir = 0.7 + rnd() * 0.12
        ph = rnd() * math.pi * 2
        sp = 0.11 + rnd() * 0.06
        lights.append({"x": x, "y": y, "r": r, "ir": ir, "ph": ph, "sp": sp})
    return {"width": width, "height": height, "rects": rects, "sdf": make_sdf(rects),
            "lights": lights, "t": 0}


def light_array(m):
    """A map's lights as rows x y r ir ph sp (the engine's and the oracle's layout)."""
    return [[l["x"], l["y"], l["r"], l["ir"], l["ph"], l["sp"]] for l in m["lights"]]


def make_sdf(rects):
    """makeSdf, map.js:91-118: signed distance + outward normal, or None."""
    def sdf(x, y):
        best, bnx, bny = math.inf, 0.0, 0.0
        for r in rects:
            cx = max(r["x"], min(x, r["x"] + r["w"]))
            cy = max(r["y"], min(y, r["y"] + r["h"]))
            dx, dy = x - cx, y - cy
            d2 = dx * dx + dy * dy
            if d2 > 1e-12:
                if d2 < best * best:
                    d = math.sqrt(d2)
                    best, bnx, bny = d, dx / d, dy / d
            else:
                dl, dr = x - r["x"], r["x"] + r["w"] - x
                dt, db = y - r["y"], r["y"] + r["h"] - y
                m = min(dl, dr, dt, db)
                d = -m
                if d < best:
                    best = d
                    if m == dl:
                        bnx, bny = -1.0, 0.0
                    elif m == dr:
                        bnx, bny = 1.0, 0.0
                    elif m == dt:
                        bnx, bny = 0.0, -1.0
                    else:
                        bnx, bny = 0.0, 1.0
        if not math.isfinite(best):
            return None
        return {"d": best, "nx": bnx, "ny": bny}

    return sdf


def find_spawn(m, clearance, rnd):
    """findSpawn, map.js:120-128."""
    for _ in range(500):
        x = clearance + rnd() * max(1, m["width"] - clearance * 2)
        y = clearance + rnd() * max(1, m["height"] - clearance * 2)
        hit = m["sdf"](x, y)
        if hit and hit["d"] >= clearance:
            return {"x": x, "y": y}
    return {"x": m["width"] * 0.5, "y": m["height"] * 0.5}


makeMap = make_map
makeSdf = make_sdf
findSpawn = find_spawn
