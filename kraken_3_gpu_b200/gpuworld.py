"""Drop-in replacement of src/gpu/gpuworld.js on the B200 C ABI.

Same surface and semantics as the reference module:

    GPU_STRIDES, isAvailable(), create(cpu, map), groupCollPoints(collPts, n),
    upload(g), uploadControls(g), packControls(cpu, consData), step(g),
    download(g) -> {maxSpeed, maxAngSpeed, nan}, mirrorInto(cpu, bodyData,
    consData), destroy(g)

``packControls``, ``mirrorInto`` and ``groupCollPoints`` are pure host
functions exactly like the reference's (gpuworld.js:189-207, 331-341,
417-456) and run without a device.  ``create``/``upload``/``step``/
``download`` call ``libkraken_b200.so``; there is no CPU fallback.  Errors
are raised as exceptions with the library's message, where the reference
throws ``Error`` (gpuworld.js:43-55, 90-97, 224-229, 269-271).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native
from .xpbd import C_GRIP, XpbdWorld, ensure_colored

BODY_STRIDE = 12
CONS_STRIDE = 20
GPU_STRIDES = {"body": BODY_STRIDE, "constraint": CONS_STRIDE, "collPt": 4, "rect": 4, "force": 4}

_U32P = C.POINTER(C.c_uint32)
_F32P = C.POINTER(C.c_float)


def isAvailable() -> bool:
    """isAvailable, gpuworld.js:30-32: a CUDA device is present."""
    return _native.lib().kr_device_count() > 0


class GpuWorld:
    """The handle ``g`` of gpuworld.js:149-166."""

    def __init__(self, handle, cpu, m, nB, nC, nP, nR):
        self.handle = handle
        self.cpu = cpu
        self.map = m
        self.nB, self.nC, self.nP, self.nR = nB, nC, nP, nR
        self.bodyData = np.zeros(nB * BODY_STRIDE, dtype=np.float32)
        self.consData = np.zeros(nC * CONS_STRIDE, dtype=np.float32)
        self.forceData = np.zeros(nB * 4, dtype=np.float32)
        self.colorWG = 1
        self.dispatches = 0


def groupCollPoints(collPts, n):
    """groupCollPoints, gpuworld.js:189-207: stable per-body grouping."""
    cnt = np.zeros(n, dtype=np.uint32)
    for i, p in enumerate(collPts):
        b = p.body
        if not (b >= 0) or b >= n:
            raise ValueError(f"collPt {i} refers to body {b} of {n}")
        cnt[b] += 1
    off = np.zeros(n, dtype=np.uint32)
    acc = 0
    for b in range(n):
        off[b] = acc
        acc += int(cnt[b])
    if acc != len(collPts):
        raise ValueError(f"collRange covers {acc} of {len(collPts)} points")
    order = np.zeros(len(collPts), dtype=np.uint32)
    cursor = off.copy()
    for i, p in enumerate(collPts):
        order[cursor[p.body]] = i
        cursor[p.body] += 1
    rng = np.concatenate([off, cnt]).astype(np.uint32)
    return {"order": order, "range": rng}


def create(cpu: XpbdWorld, m, wgslSource=None, device=None) -> GpuWorld:
    """create + writeStatic, gpuworld.js:34-171, 209-247.  ``wgslSource`` and
    ``device`` are accepted for signature parity and ignored."""
    ensure_colored(cpu)
    nB, nC, nP, nR = cpu.n, len(cpu.constraints), len(cpu.collPts), len(m["rects"])
    rect_data = np.zeros(max(nR, 1) * 4, dtype=np.float32)
    for i, r in enumerate(m["rects"]):
        rect_data[4 * i: 4 * i + 4] = (r["x"], r["y"], r["w"], r["h"])
    grouped = groupCollPoints(cpu.collPts, nB)
    coll_data = np.zeros(max(nP, 1) * 4, dtype=np.float32)
    coll_u = coll_data.view(np.uint32)
    for o4, idx in enumerate(grouped["order"]):
        p = cpu.collPts[int(idx)]
        coll_u[4 * o4] = p.body
        coll_data[4 * o4 + 1: 4 * o4 + 4] = (p.lx, p.ly, p.r)
    rng = np.ascontiguousarray(grouped["range"], dtype=np.uint32)
    params = _native.SolverParams(cpu.h, cpu.substeps, cpu.iterations, cpu.linDrag, cpu.angDrag,
                                  cpu.maxSpeed, cpu.maxAngSpeed)
    h = C.c_void_p()
    L = _native.lib()
    rc = L.kr_create(C.byref(params), nB, nC, rect_data.ctypes.data_as(_F32P), nR,
                     coll_u.ctypes.data_as(_U32P), nP, rng.ctypes.data_as(_U32P), C.byref(h))
    _native.check(rc, None)
    return GpuWorld(h, cpu, m, nB, nC, nP, nR)


def upload(g: GpuWorld):
    """upload, gpuworld.js:250-298: CPU state -> device (overwrites it)."""
    cpu = g.cpu
    n = cpu.n
    bd = g.bodyData.reshape(n, BODY_STRIDE)
    for col, name in enumerate(("px", "py", "ppx", "ppy", "vx", "vy", "ang", "angP", "av",
                                "im", "ii")):
        bd[:, col] = getattr(cpu, name)[:n]
    bd[:, 11] = 0
    fd = g.forceData.reshape(n, 4)
    fd[:, 0] = cpu.fx[:n]
    fd[:, 1] = cpu.fy[:n]
    fd[:, 2] = cpu.tq[:n]
    fd[:, 3] = 0
    cd = g.consData
    cu = cd.view(np.uint32)
    for k, c in enumerate(cpu.constraints):
        o = k * CONS_STRIDE
        if c.a >= n or (c.b >= 0 and c.b >= n):
            raise IndexError(f"Constraint {k}: body index {c.a}/{c.b} outside of {n} "
                             "(an out-of-bounds read in the kernel)")
        cu[o] = c.a
        cu[o + 1] = c.b if c.b >= 0 else 0xFFFFFFFF
        cu[o + 2] = c.type
        cu[o + 3] = c.owner & 0xFFFFFFFF
        cd[o + 4] = c.lax
        cd[o + 5] = c.lay
        cd[o + 6] = c.lbx
        cd[o + 7] = c.lby
        cd[o + 8] = c.compliance
        cd[o + 9] = c.rest
        cd[o + 10] = c.target
        cd[o + 11] = c.minAngle
        cd[o + 12] = c.maxAngle
        cd[o + 13] = c.lambdaX or 0
        cd[o + 14] = c.lambdaY or 0
        cd[o + 15] = c.lambda_
        cd[o + 16] = min(c.breakForce, 1e30) if math.isfinite(c.breakForce) else 1e30
        cu[o + 17] = 1 if c.broken else 0
        cu[o + 18] = 0
        cu[o + 19] = 0
    ci = np.zeros(33, dtype=np.uint32)
    max_cnt = 0
    for c in range(16):
        ci[c] = cpu.colorOff[c]
        ci[16 + c] = cpu.colorCnt[c]
        max_cnt = max(max_cnt, int(cpu.colorCnt[c]))
    ci[32] = max(1, math.ceil(max_cnt / 64))
    g.colorWG = int(ci[32])
    rc = _native.lib().kr_upload(g.handle, g.bodyData.ctypes.data_as(_F32P),
                                 cu.ctypes.data_as(_U32P), g.forceData.ctypes.data_as(_F32P),
                                 ci.ctypes.data_as(_U32P))
    _native.check(rc, g.handle)


def packControls(cpu: XpbdWorld, consData: np.ndarray):
    """packControls, gpuworld.js:331-341: control fields into the 80 B blocks
    (compliance o+8, target o+10, lbx/lby o+6/7, breakForce o+16 with
    inf -> 1e30, broken o+17 through the u32 view)."""
    cu = consData.view(np.uint32)
    for k, c in enumerate(cpu.constraints):
        o = k * CONS_STRIDE
        consData[o + 6] = c.lbx
        consData[o + 7] = c.lby
        consData[o + 8] = c.compliance
        consData[o + 10] = c.target
        consData[o + 16] = min(c.breakForce, 1e30) if math.isfinite(c.breakForce) else 1e30
        cu[o + 17] = 1 if c.broken else 0


def uploadControls(g: GpuWorld):
    """uploadControls, gpuworld.js:312-315."""
    packControls(g.cpu, g.consData)
    rc = _native.lib().kr_upload_controls(g.handle, g.consData.view(np.uint32).ctypes.data_as(_U32P))
    _native.check(rc, g.handle)


def step(g: GpuWorld, n: int = 1):
    """step, gpuworld.js:374-382: one env step (substeps + gripBreak) per call."""
    rc = _native.lib().kr_step(g.handle, n)
    _native.check(rc, g.handle)
    g.dispatches += n


def download(g: GpuWorld):
    """download, gpuworld.js:385-396: device -> CPU world via mirrorInto."""
    bd = np.zeros(g.nB * BODY_STRIDE, dtype=np.float32)
    cd = np.zeros(g.nC * CONS_STRIDE, dtype=np.float32)
    rc = _native.lib().kr_download(g.handle, bd.ctypes.data_as(_F32P),
                                   cd.view(np.uint32).ctypes.data_as(_U32P))
    _native.check(rc, g.handle)
    return mirrorInto(g.cpu, bd, cd)


def mirrorInto(cpu: XpbdWorld, bodyData: np.ndarray, consData: np.ndarray):
    """mirrorInto, gpuworld.js:417-456: px, py, vx, vy, ang, av of every body,
    lambda and broken of every constraint, lambdaX/Y and force of grips."""
    cu = consData.view(np.uint32)
    n = cpu.n
    bd = bodyData.reshape(-1, BODY_STRIDE)[:n].astype(np.float64)
    px, py, vx, vy, ang, av = bd[:, 0], bd[:, 1], bd[:, 4], bd[:, 5], bd[:, 6], bd[:, 8]
    cpu.px[:n] = px
    cpu.py[:n] = py
    cpu.vx[:n] = vx
    cpu.vy[:n] = vy
    cpu.ang[:n] = ang
    cpu.av[:n] = av
    # JS `if (s2 > maxS2)` skips NaN; so does this
    s2 = vx * vx + vy * vy
    s2 = np.where(np.isnan(s2), 0.0, s2)
    aa = np.abs(av)
    aa = np.where(np.isnan(aa), 0.0, aa)
    max_s2 = max(0.0, float(np.max(s2))) if n else 0.0
    max_ang_speed = max(0.0, float(np.max(aa))) if n else 0.0
    bad = ~(np.isfinite(px) & np.isfinite(py) & np.isfinite(vx) & np.isfinite(vy) & np.isfinite(ang))
    nan = int(np.count_nonzero(bad))
    max_speed = math.sqrt(max_s2)
    inv_h = 1 / cpu.h
    for k, c in enumerate(cpu.constraints):
        o = k * CONS_STRIDE
        c.lambda_ = float(consData[o + 15])
        c.broken = int(cu[o + 17]) != 0
        if c.type == C_GRIP:
            c.lambdaX = float(consData[o + 13])
            c.lambdaY = float(consData[o + 14])
            c.force = math.hypot(c.lambdaX, c.lambdaY) * inv_h
    cpu.stats["maxSpeed"] = max_speed
    cpu.stats["maxAngSpeed"] = max_ang_speed
    cpu.stats["nan"] = nan
    return {"maxSpeed": max_speed, "maxAngSpeed": max_ang_speed, "nan": nan}


def destroy(g: GpuWorld):
    """destroy, gpuworld.js:466-472: frees the device buffers (errors ignored)."""
    if g is None or not getattr(g, "handle", None):
        return
    try:
        _native.lib().kr_destroy(g.handle)
    finally:
        g.handle = None


def islands(g: GpuWorld):
    """(connected components, constraint levels of the largest) of the last upload."""
    n, lv = C.c_int32(), C.c_int32()
    _native.check(_native.lib().kr_world_islands(g.handle, C.byref(n), C.byref(lv)), g.handle)
    return n.value, lv.value
