"""GPU parity of the plain per-step kernel through the gpuworld drop-in.

Bars (tolerances written in the tests):
  * vs the f32 oracle (tools/f32solver.mjs restated): <= 4 ulp per body
    coordinate after 1 step; the kernel follows the same op order, so the
    tests also record that it is bit-identical.
  * vs the FP64 oracle (src/physics/xpbd.js restated): <= 1e-3 px after 1
    step, <= 1e-2 px after 60 steps, identical attach / release / break event
    sequences over those 60 steps.
Host loop = the reference's hybrid trainer (gputrain.js:72-128): CPU reflex
on the mirrored state, uploadControls, step, download.
"""
import math

import numpy as np
import pytest

from kraken_3_gpu_b200 import core, gpuworld, kraken, world_map, xpbd
from oracle import binding as ob
from tests.scenarios import TONE, ControlStream, ulp_distance

pytestmark = pytest.mark.gpu


class Hybrid:
    """The package's world on the GPU, driven like gputrain.gpuTrainStep."""

    def __init__(self, seed, creatures, arms=6, segs=7):
        self.sim = core.create_sim(seed=seed, creatures=creatures, arms=arms, segsPerArm=segs)
        self.w = self.sim["world"]
        self.g = gpuworld.create(self.w, self.sim["map"])
        gpuworld.upload(self.g)
        # mirror the device's f32 state once, as the f32 oracle's roundState does,
        # so the first reflex attaches from the same state on both sides
        gpuworld.download(self.g)

    def control(self, ci, targets, adhesion):
        core.apply_control_motors(self.sim["creatures"][ci], TONE, targets, adhesion)

    def step(self):
        gpuworld.uploadControls(self.g)
        gpuworld.step(self.g)
        return gpuworld.download(self.g)

    def grips(self, ci):
        return [a.grip.broken for a in self.sim["creatures"][ci].arms]

    def close(self):
        gpuworld.destroy(self.g)


def _oracle(seed, creatures, f32, arms=6, segs=7):
    o = ob.Sim(seed=seed, creatures=creatures, arms=arms, segs=segs)
    if f32:
        o.world.f32ify()
        o.world.round_state()
    return o


def _events(prev, cur, step, ci):
    ev = []
    for a, (p, c) in enumerate(zip(prev, cur)):
        if p != c:
            ev.append((step, ci, a, "attach" if not c else "detach"))
    return ev


def test_one_step_vs_f32_oracle_default_body():
    h = _oracle(1, 1, True)
    g = Hybrid(1, 1)
    try:
        cs = ControlStream()
        t, a = cs.at(0)
        g.control(0, t, a)
        h.apply_control_motors(0, TONE, t, a)
        g.step()
        h.step32()
        n = g.w.n
        for name in ("px", "py", "vx", "vy", "ang", "av"):
            u = ulp_distance(getattr(g.w, name)[:n].astype(np.float32),
                             h.world.arr(name).astype(np.float32))
            assert u.max() <= 4, name
            assert u.max() == 0, f"{name}: not bit-identical (max {u.max()} ulp)"
    finally:
        g.close()


@pytest.mark.parametrize("arms,segs,seed", [(4, 5, 3), (8, 9, 5), (6, 7, 17)])
def test_ten_steps_vs_f32_oracle_bodies(arms, segs, seed):
    creatures = 3
    h = _oracle(seed, creatures, True, arms, segs)
    g = Hybrid(seed, creatures, arms, segs)
    try:
        streams = [ControlStream(arms, segs, seed=100 + c) for c in range(creatures)]
        worst = 0
        for s in range(10):
            for c in range(creatures):
                t, a = streams[c].at(s)
                g.control(c, t, a)
                h.apply_control_motors(c, TONE, t, a)
            g.step()
            h.step32()
            n = g.w.n
            for name in ("px", "py", "ang"):
                u = ulp_distance(getattr(g.w, name)[:n].astype(np.float32),
                                 h.world.arr(name).astype(np.float32))
                worst = max(worst, int(u.max()))
            if s == 0:
                assert worst <= 4
        assert worst == 0, f"max {worst} ulp after 10 steps"
    finally:
        g.close()


def test_sixty_steps_vs_fp64_oracle_with_events():
    """Config 0: default body on map seed 1, controls from mulberry32(0)."""
    h = _oracle(1, 1, False)
    g = Hybrid(1, 1)
    try:
        cs = ControlStream(seed=0)
        ev_g, ev_h = [], []
        prev_g = g.grips(0)
        oc = h.creatures[0]
        prev_h = [oc.grip(a).broken for a in range(6)]
        for s in range(60):
            t, a = cs.at(s)
            g.control(0, t, a)
            h.apply_control_motors(0, TONE, t, a)
            cur_g, cur_h = g.grips(0), [oc.grip(a).broken for a in range(6)]
            ev_g += _events(prev_g, cur_g, s, 0)
            ev_h += _events(prev_h, cur_h, s, 0)
            g.step()
            h.step()
            prev_g, prev_h = cur_g, cur_h
            cur_g, cur_h = g.grips(0), [oc.grip(a).broken for a in range(6)]
            ev_g += _events(prev_g, cur_g, s, 1)
            ev_h += _events(prev_h, cur_h, s, 1)
            prev_g, prev_h = cur_g, cur_h
            n = g.w.n
            d = max(np.max(np.abs(g.w.px[:n] - h.world.px)), np.max(np.abs(g.w.py[:n] - h.world.py)))
            if s == 0:
                assert d <= 1e-3, f"step 1: {d} px"
        assert d <= 1e-2, f"step 60: {d} px"
        assert ev_g == ev_h
        assert len(ev_g) > 0, "scenario produced no grip events"
    finally:
        g.close()


def test_batch_256_creatures_vs_f32_oracle():
    h = _oracle(9, 256, True)
    g = Hybrid(9, 256)
    try:
        streams = [ControlStream(seed=1000 + c) for c in range(256)]
        for s in range(4):
            for c in range(256):
                t, a = streams[c].at(s)
                g.control(c, t, a)
                h.apply_control_motors(c, TONE, t, a)
            g.step()
            h.step32()
        n = g.w.n
        for name in ("px", "py", "ang", "vx", "vy", "av"):
            u = ulp_distance(getattr(g.w, name)[:n].astype(np.float32),
                             h.world.arr(name).astype(np.float32))
            assert u.max() <= 4, name
        ni, lv = gpuworld.islands(g.g)
        assert ni == 256 and lv == 12
    finally:
        g.close()


def _build_world(n, seed):
    """gpu.html:200-211 buildWorld on the package's builders."""
    m = world_map.make_map(1440, 810, seed=seed)
    rnd = world_map.mulberry32(seed ^ 0x5BF03635)
    w = xpbd.XpbdWorld(substeps=2, iterations=4, h=1 / 120, maxSpeed=360, maxAngSpeed=18)
    w.sdf = m["sdf"]
    ks = []
    for _ in range(n):
        sp = world_map.find_spawn(m, kraken.ARM_REACH + 20, rnd)
        ks.append(kraken.spawn_kraken(w, sp["x"], sp["y"], rnd() * math.pi * 2))
    return w, m, ks


def test_g1_passive_fixpoint():
    # gpu.html:223-268: 240 + 2160 steps without drive, displacement exactly 0
    w, m, ks = _build_world(4, 11)
    spawn = [(w.px[k.mantle], w.py[k.mantle]) for k in ks]
    g = gpuworld.create(w, m)
    try:
        gpuworld.upload(g)
        gpuworld.step(g, 240)
        st = gpuworld.download(g)
        path = sum(math.hypot(w.px[k.mantle] - sx, w.py[k.mantle] - sy) for k, (sx, sy) in zip(ks, spawn))
        gpuworld.step(g, 2160)
        st2 = gpuworld.download(g)
        path2 = sum(math.hypot(w.px[k.mantle] - sx, w.py[k.mantle] - sy) for k, (sx, sy) in zip(ks, spawn))
        assert path < 0.05 and path2 - path < 0.01
        assert st2["maxSpeed"] < 0.05 and st["nan"] == 0
    finally:
        gpuworld.destroy(g)


def test_g3_grip_pull_gate():
    # gpu.html:302-339: GPU pull within 30% of the CPU's 70.328 px, same break state
    w, m, ks = _build_world(1, 31)
    k, arm = ks[0], ks[0].arms[0]
    kraken.attach_grip(w, arm, kraken.adhesion_to_break_force(1.0))
    anchor = kraken.tip_position(w, arm)
    start = math.hypot(w.px[k.mantle] - anchor["x"], w.py[k.mantle] - anchor["y"])
    g = gpuworld.create(w, m)
    try:
        gpuworld.upload(g)
        comp = kraken.tone_to_compliance(1.0)
        min_d = start
        for _ in range(600):
            for mm in arm.motors:
                mm.compliance = comp
            arm.motors[0].target = 0
            for j in range(1, len(arm.motors)):
                arm.motors[j].target = kraken.BODY["jointLimit"] * 0.98
            for a in k.arms[1:]:
                for mm in a.motors:
                    mm.compliance = kraken.tone_to_compliance(0.2)
                    mm.target = 0
            arm.grip.breakForce = kraken.adhesion_to_break_force(1.0)
            gpuworld.uploadControls(g)
            gpuworld.step(g)
            gpuworld.download(g)
            if arm.grip.broken:
                break
            min_d = min(min_d, math.hypot(w.px[k.mantle] - anchor["x"], w.py[k.mantle] - anchor["y"]))
        pulled = start - min_d
        assert not arm.grip.broken
        assert abs(pulled - 70.328) / 70.328 < 0.30 and pulled > 0.5 * 70.328
        assert abs(pulled - 70.328) < 0.5  # f32 vs f64: the reference's GPU got 70.339
    finally:
        gpuworld.destroy(g)


def test_g5_determinism_under_load():
    def run():
        w, m, ks = _build_world(4, 59)
        g = gpuworld.create(w, m)
        try:
            gpuworld.upload(g)
            for k in ks:
                for arm in k.arms:
                    for mm in arm.motors:
                        mm.compliance = kraken.tone_to_compliance(0.8)
                        mm.target = 0.5
            gpuworld.uploadControls(g)
            gpuworld.step(g, 300)
            gpuworld.download(g)
            return w.px[: w.n].tobytes() + w.py[: w.n].tobytes()
        finally:
            gpuworld.destroy(g)
    assert run() == run()


def test_state_errors():
    from kraken_3_gpu_b200 import _native
    sim = core.create_sim(seed=1, creatures=1)
    g = gpuworld.create(sim["world"], sim["map"])
    try:
        with pytest.raises(_native.KrError) as e:
            gpuworld.step(g)
        assert e.value.code == _native.KR_ERR_STATE
        sim["world"].constraints[3].b = 10_000
        with pytest.raises(IndexError):
            gpuworld.upload(g)
    finally:
        gpuworld.destroy(g)
