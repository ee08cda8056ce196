"""The reference's hybrid training loop over the drop-in, for many creatures
of one body shape at once (src/sim/gputrain.js:72-128): per env step
applyControl with the suction-cup reflex on the mirrored f32 state
(src/sim/core.js:183-220), uploadControls, one step, download and mirror --
through the drop-in C ABI (include/kraken_b200.h) with host buffers.

The host side runs over numpy arrays instead of per-creature objects: each
creature's control stream (mulberry32, src/world/map.js:11-20, redrawn every
6 env steps, held as f32 like the controls of a Float32Array), the clamped
motor targets and the tone's compliance, the reflex (slip gate, attach at the
tip point, break force, release) and packControls' fields
(src/gpu/gpuworld.js:331-341) of the motors and grips.  Driven this way the
drop-in computes exactly what the batched engine computes with its reflex
on the device (the GPU tests check it bit for bit).
"""
from __future__ import annotations

import ctypes as C

import numpy as np


class HybridLoop:
    """w: a workload of one body shape on one map (workloads.uniform);
    stream_ptr: the CUDA stream (cudaStream_t as int) the world runs on.
    step(ev=None) advances every creature one env step (ev: a pair of CUDA
    events recorded around the kernel launch)."""

    def __init__(self, w, stream_ptr):
        from . import _native, core, gpuworld, kraken
        self.n = w.n
        self.sim = core.create_sim(seed=1, creatures=w.n, poses=list(zip(w.x, w.y, w.angle)))
        world, crs = self.sim["world"], self.sim["creatures"]
        self.g = gpuworld.create(world, self.sim["map"])
        gpuworld.upload(self.g)
        self.L, self.h = _native.lib(), self.g.handle
        _native.check(self.L.kr_set_stream(self.h, C.c_void_p(stream_ptr)), self.h)
        k_of = {id(c): k for k, c in enumerate(world.constraints)}
        self.motors = np.array([[k_of[id(m)] for a in c.arms for m in a.motors] for c in crs])
        self.grips = np.array([[k_of[id(a.grip)] for a in c.arms] for c in crs])
        self.tips = np.array([[a.tip for a in c.arms] for c in crs])
        self.A, self.S = len(crs[0].arms), len(crs[0].arms[0].motors)
        B = kraken.BODY
        self.lim = np.where(np.arange(self.A * self.S) % self.S == 0, B["shoulderLimit"], B["jointLimit"])
        self.half_seg = B["segLen"] * 0.5
        self.cons = self.g.consData.reshape(-1, 20)
        self.consu = self.g.consData.view(np.uint32).reshape(-1, 20)
        self.body = self.g.bodyData.reshape(-1, 12)
        self.comp = kraken.tone_to_compliance(0.5)
        self.rng = np.ascontiguousarray(w.seed, dtype=np.uint32).copy()
        self.targets = np.zeros((self.n, self.A * self.S))
        self.adh = np.zeros((self.n, self.A))
        self.cd = np.zeros((self.n, self.A))
        self.dt = world.h * world.substeps
        self.cp = self.g.consData.view(np.uint32).ctypes.data_as(C.POINTER(C.c_uint32))
        self.bp = self.g.bodyData.ctypes.data_as(C.POINTER(C.c_float))
        self.t = 0
        self._check(self.L.kr_download(self.h, self.bp, self.cp))  # the mirrored f32 state

    def _check(self, rc):
        from . import _native
        _native.check(rc, self.h)

    def _draw(self):
        r = np.empty((self.n, self.A * (self.S + 1)))
        s = self.rng
        for d in range(r.shape[1]):
            s = s + np.uint32(0x6D2B79F5)
            t = (s ^ (s >> np.uint32(15))) * (s | np.uint32(1))
            t ^= t + (t ^ (t >> np.uint32(7))) * (t | np.uint32(61))
            r[:, d] = (t ^ (t >> np.uint32(14))) / 4294967296.0
        self.rng = s
        r = r.reshape(self.n, self.A, self.S + 1)
        # held as f32, as the controls of a Float32Array (the engine's control record)
        self.targets = (r[:, :, :self.S] * 2 - 1).astype(np.float32).astype(np.float64).reshape(self.n, -1)
        self.adh = r[:, :, self.S].astype(np.float32).astype(np.float64)

    def control(self):
        """applyControl for every creature on the mirrored state, packed."""
        if self.t % 6 == 0:
            self._draw()
        self.cons[self.motors, 8] = self.comp  # every step, as packControls writes it
        self.cons[self.motors, 10] = np.clip(self.targets, -self.lim, self.lim)
        adh = np.clip(self.adh, 0.0, 1.0)
        self.cd = np.where(self.cd > 0, self.cd - self.dt, self.cd)
        broken = self.consu[self.grips, 17] != 0
        tb = self.body[self.tips].astype(np.float64)
        cand = broken & (adh > 0.08) & (self.cd <= 0)
        att = cand & (np.hypot(tb[..., 4], tb[..., 5]) < 150.0)
        self.cd = np.where(cand & ~att, 0.05, self.cd)
        held = ~broken
        ga = self.grips[att]
        self.cons[ga, 6] = tb[..., 0][att] + self.half_seg * np.cos(tb[..., 6][att])
        self.cons[ga, 7] = tb[..., 1][att] + self.half_seg * np.sin(tb[..., 6][att])
        upd = att | held
        self.cons[self.grips[upd], 16] = (40.0 + 860.0 * adh)[upd]
        nb = broken & ~att | (held & (adh < 0.04))
        self.consu[self.grips, 17] = nb.astype(np.uint32)

    def step(self, ev=None):
        self.control()
        self._check(self.L.kr_upload_controls(self.h, self.cp))
        if ev is not None:
            ev[0].record()
        self._check(self.L.kr_step(self.h, 1))
        if ev is not None:
            ev[1].record()
        self._check(self.L.kr_download(self.h, self.bp, self.cp))
        self.t += 1

    def close(self):
        from . import gpuworld
        gpuworld.destroy(self.g)
