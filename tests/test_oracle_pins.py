"""Pins of the CPU oracle against the reference's own quoted results.

The reference publishes no per-particle golden vectors; its harness
(tools/harness.js) and README quote scalar results of seeded scenarios.
These tests rebuild the same scenarios on the oracle (the C restatement of
src/physics/xpbd.js, src/world/map.js, src/body/kraken.js, src/sim/core.js)
and compare with those numbers.
"""
import math

import numpy as np
import pytest

from oracle import binding as ob

JOINT = math.pi * 0.42
SHOULDER = math.pi * 0.62


def test_map_rect_counts():
    # map seed 1: 24 rects (probe of map.js:22-71); seed 5: 18 rects
    # (harness.js:1212-1216 "18 Rechtecke x 6 Lagen" -> 128 poses with 20 sim poses)
    assert len(ob.make_map_rects(seed=1)) == 24
    assert len(ob.make_map_rects(seed=5)) == 18


def test_colour_classes_default_body():
    # createSim colouring (core.js:45-58) + groupConstraintsByColor (core.js:276-288)
    s = ob.Sim(seed=1, creatures=1)
    off, cnt = s.world.color_info()
    assert cnt == [24, 19, 20, 19, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0]
    assert s.world.n == 43 and s.world.nC == 90 and s.world.nP == 92


def test_mirror_field_sizes():
    # harness mirror-fields: createSim(seed 31, 2 creatures) -> 86 bodies, 180 constraints
    s = ob.Sim(seed=31, creatures=2)
    assert s.world.n == 86 and s.world.nC == 180


def _build_world(n, seed):
    """gpu.html:200-211 buildWorld (creation-order constraint list)."""
    rects = ob.make_map_rects(seed=seed)
    rng = ob.Rng(seed ^ 0x5BF03635)
    w = ob.World()
    w.set_rects(rects)
    ks = []
    for _ in range(n):
        x, y = ob.find_spawn(rects, 1440, 810, ob.arm_reach() + 20, rng)
        ks.append(w.spawn_kraken(x, y, rng() * math.pi * 2))
    return w, rects, ks


def test_g3_grip_pull_cpu_70_328():
    # gpu.html:302-339 (G3, CPU run); README:475 "G3 Zugweg 70.328 CPU"
    w, _, ks = _build_world(1, 31)
    k = ks[0]
    k.attach_grip(0, ob.adhesion_to_break_force(1.0))
    ax, ay = k.tip_position(0)
    start = math.hypot(w.px[k.mantle] - ax, w.py[k.mantle] - ay)
    min_d = start
    for _ in range(600):
        for m in k.motors[0]:
            w.con(m).compliance = ob.tone_to_compliance(1.0)
        w.con(k.motors[0][0]).target = 0
        for j in range(1, len(k.motors[0])):
            w.con(k.motors[0][j]).target = JOINT * 0.98
        for a in range(1, 6):
            for m in k.motors[a]:
                w.con(m).compliance = ob.tone_to_compliance(0.2)
                w.con(m).target = 0
        k.grip(0).breakForce = ob.adhesion_to_break_force(1.0)
        w.step()
        if k.grip(0).broken:
            break
        min_d = min(min_d, math.hypot(w.px[k.mantle] - ax, w.py[k.mantle] - ay))
    assert not k.grip(0).broken
    assert f"{start - min_d:.3f}" == "70.328"


def test_grip_pull_harness_70_6_px_72pct():
    # harness.js:165-206; README:163 "70.6 px = 72 %"
    rows = []
    for tone in (0.3, 0.65, 1.0):
        s = ob.Sim(seed=11, creatures=1)
        c, w = s.creatures[0], s.world
        c.attach_grip(0, ob.adhesion_to_break_force(1.0))
        ax, ay = c.tip_position(0)
        start = math.hypot(w.px[c.mantle] - ax, w.py[c.mantle] - ay)
        min_d = start
        for _ in range(600):
            cu = np.zeros(6)
            cu[0] = JOINT * 0.98
            ad = np.zeros(6)
            ad[0] = 1
            s.apply_control(0, tone, np.zeros(6), cu, ad)
            s.step()
            if c.grip(0).broken:
                break
            min_d = min(min_d, math.hypot(w.px[c.mantle] - ax, w.py[c.mantle] - ay))
        rows.append((start - min_d, (start - min_d) / start * 100))
    best = max(rows, key=lambda r: r[1])
    assert f"{best[0]:.1f}" == "70.6" and f"{best[1]:.0f}" == "72"


def test_passive_exact_rest():
    # harness.js:45-57: 960 steps without drive -> pathLen and displacement < 1e-9
    s = ob.Sim(seed=7, creatures=1)
    c, w = s.creatures[0], s.world
    x0, y0 = w.px[c.mantle], w.py[c.mantle]
    for _ in range(960):
        s.step()
    assert math.hypot(w.px[c.mantle] - x0, w.py[c.mantle] - y0) < 1e-9
    assert w.stats["nan"] == 0


def _viol_pins(w):
    worst = 0.0
    px, py, ang = w.px, w.py, w.ang
    for c in w.constraints:
        if c.type != ob.C_PIN or c.broken:
            continue
        A, B = c.a, c.b
        ca, sa = math.cos(ang[A]), math.sin(ang[A])
        gax, gay = px[A] + c.lax * ca - c.lay * sa, py[A] + c.lax * sa + c.lay * ca
        if B >= 0:
            cb, sb = math.cos(ang[B]), math.sin(ang[B])
            gbx, gby = px[B] + c.lbx * cb - c.lby * sb, py[B] + c.lbx * sb + c.lby * cb
        else:
            gbx, gby = c.lbx, c.lby
        worst = max(worst, math.hypot(gax - gbx, gay - gby))
    return worst


def test_slack_fixpoint_and_corrects():
    # harness.js:60-115; README:142 "0.050 px -> 1.95e-3 px"
    rects = ob.make_map_rects(seed=5)
    sp = ob.find_spawn(rects, 1440, 810, ob.arm_reach() + 20, ob.Rng(9))
    w1 = ob.World()
    w1.set_rects(rects)
    k1 = w1.spawn_kraken(sp[0], sp[1], 0.4)
    w1.px[k1.segs[0][1]] += 2e-3 * 0.4
    p0, q0, a0 = w1.px.copy(), w1.py.copy(), w1.ang.copy()
    for _ in range(240):
        w1.step()
    moved = max(np.max(np.hypot(w1.px - p0, w1.py - q0)), np.max(np.abs(w1.ang - a0)))
    assert moved == 0 and w1.stats["maxSpeed"] == 0 and w1.stats["maxAngSpeed"] == 0

    w2 = ob.World()
    w2.set_rects(rects)
    k2 = w2.spawn_kraken(sp[0], sp[1], 0.4)
    w2.px[k2.segs[0][1]] += 0.05
    before = _viol_pins(w2)
    for _ in range(240):
        w2.step()
    after = _viol_pins(w2)
    assert before > 0.04 and after < 0.01
    # the README quotes 1.95e-3; the restatement lands at 1.97e-3 (both are
    # just under the 2e-3 dead band, where V8-vs-glibc last-bit trig decides)
    assert after == pytest.approx(1.95e-3, rel=0.02)


def test_break_and_hold():
    # harness.js:209-251 pass criteria (weak grip breaks, strong grip holds)
    def run(adh):
        s = ob.Sim(seed=13, creatures=1)
        c = s.creatures[0]
        c.attach_grip(0, ob.adhesion_to_break_force(adh))
        broke = False
        for _ in range(400):
            sh = np.array([0.0] + [(1 if j % 2 else -1) * SHOULDER * 0.8 for j in range(1, 6)])
            ad = np.zeros(6)
            ad[0] = adh
            s.apply_control(0, 1.0, sh, np.full(6, JOINT * 0.9), ad)
            s.step()
            if c.grip(0).broken:
                broke = True
                break
        return broke, c.grip(0).force
    broke, peak = run(0.05)
    assert broke and peak > ob.adhesion_to_break_force(0.05)
    held, _ = run(1.0)
    assert not held


def test_mass_ratios():
    # harness.js:290-305; README:170-171 "11.1:1", "1.78:1"
    s = ob.Sim(seed=5, creatures=1)
    w, c = s.world, s.creatures[0]
    mm = 1 / w.im[c.mantle]
    ms = [1 / w.im[b] for arm in c.segs for b in arm]
    assert f"{mm / min(ms):.1f}" == "11.1"
    assert f"{max(ms) / min(ms):.2f}" == "1.78"


def test_determinism():
    # harness.js:308-326
    def run(seed):
        s = ob.Sim(seed=seed, creatures=2)
        for i in range(300):
            for ci in range(2):
                s.apply_control(ci, 0.8, [math.sin(i * 0.1 + j) * 0.6 for j in range(6)],
                                [math.sin(i * 0.2 + j) * 0.7 for j in range(6)], [0.6] * 6)
            s.step()
        w = s.world
        return [(w.px[c.mantle], w.py[c.mantle], w.ang[c.mantle]) for c in s.creatures]
    assert run(42) == run(42)
    assert run(42) != run(43)


def test_coll_grouping_26356_contacts():
    # harness.js:1197-1273; README:161 "128 Posen, 26 356 Kontakte, Delta = 0"
    s = ob.Sim(seed=5, creatures=3)
    w, rects = s.world, s.rects
    poses = []
    for r in rects:
        for v in range(6):
            i = np.arange(w.n)
            u = ((i + v * 7) % 10) / 10
            px = r[0] + r[2] * (u if v % 2 else 0.5) + (v % 3) - 1
            py = r[1] + r[3] * (0.5 if v % 2 else u) + ((v >> 1) % 3) - 1
            px = np.broadcast_to(px, (w.n,)).astype(np.float64)
            py = np.broadcast_to(py, (w.n,)).astype(np.float64)
            ang = np.array([math.fmod(k * 0.7 + v * 1.1, 6.283) for k in range(w.n)])
            poses.append((px, py, ang))
    rnd = ob.Rng(4242)
    for _ in range(20):
        for ci in range(3):
            tone = 0.2 + 0.6 * rnd()
            sh, cu, ad = [], [], []
            for _a in range(6):
                sh.append(rnd() * 2 - 1)
                cu.append(rnd() * 2 - 1)
                ad.append(rnd())
            s.apply_control(ci, tone, sh, cu, ad)
        s.step()
        poses.append((w.px.copy(), w.py.copy(), w.ang.copy()))
    assert len(poses) == 128
    pts = w.coll_pts()
    by_body = [[] for _ in range(w.n)]
    for p in pts:
        by_body[p[0]].append(p)
    im = w.im.copy()
    contacts, max_err = 0, 0.0
    for px, py, ang in poses:
        w.px[:] = px
        w.py[:] = py
        w.ang[:] = ang
        w.ppx[:] = px
        w.ppy[:] = py
        w.angP[:] = ang
        w.solve_collisions()
        ref_x, ref_y = w.ppx.copy(), w.ppy.copy()
        for b in range(w.n):
            if im[b] == 0:
                continue
            x, y = px[b], py[b]
            for _b, lx, ly, r in by_body[b]:
                ca, sa = math.cos(ang[b]), math.sin(ang[b])
                hit = ob.sdf(rects, x + lx * ca - ly * sa, y + lx * sa + ly * ca)
                if hit is None:
                    continue
                pen = r - hit[0]
                if pen <= 2e-3:
                    continue
                x += hit[1] * pen
                y += hit[2] * pen
                contacts += 1
            max_err = max(max_err, abs(x - ref_x[b]), abs(y - ref_y[b]))
    assert contacts == 26356 and max_err == 0
