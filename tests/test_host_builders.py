"""Host-side builders of the package against the oracle's builders (bit-exact).

The package rebuilds map.js / kraken.js / core.js on the host (Python); the
oracle restates the same files in C.  Both must produce identical worlds,
since the GPU parity tests run the package's world against the oracle's.
"""
import math

import numpy as np
import pytest

from kraken_3_gpu_b200 import core, kraken, world_map, xpbd
from oracle import binding as ob


def test_mulberry32_stream():
    r1 = world_map.mulberry32(0x5BF03635 ^ 31)
    r2 = ob.Rng(0x5BF03635 ^ 31)
    assert [r1() for _ in range(1000)] == [r2() for _ in range(1000)]


@pytest.mark.parametrize("seed", [1, 5, 7, 31, 12345])
def test_make_map_matches(seed):
    m = world_map.make_map(1440, 810, seed=seed)
    got = np.array([[r["x"], r["y"], r["w"], r["h"]] for r in m["rects"]])
    assert np.array_equal(got, ob.make_map_rects(seed=seed))


def test_sdf_matches():
    m = world_map.make_map(1440, 810, seed=1)
    rects = ob.make_map_rects(seed=1)
    rnd = world_map.mulberry32(3)
    for _ in range(2000):
        x, y = rnd() * 1500 - 30, rnd() * 870 - 30
        a, b = m["sdf"](x, y), ob.sdf(rects, x, y)
        assert (a is None) == (b is None)
        if a:
            assert (a["d"], a["nx"], a["ny"]) == b


@pytest.mark.parametrize("seed,creatures,arms,segs", [(1, 1, 6, 7), (7, 3, 6, 7), (11, 2, 4, 5),
                                                       (3, 2, 8, 9), (5, 1, 5, 6)])
def test_create_sim_matches(seed, creatures, arms, segs):
    sim = core.create_sim(seed=seed, creatures=creatures, arms=arms, segsPerArm=segs)
    w = sim["world"]
    o = ob.Sim(seed=seed, creatures=creatures, arms=arms, segs=segs)
    ow = o.world
    assert w.n == ow.n and len(w.constraints) == ow.nC and len(w.collPts) == ow.nP
    for name in ("px", "py", "ppx", "ppy", "vx", "vy", "ang", "angP", "av", "im", "ii"):
        assert np.array_equal(getattr(w, name)[: w.n], ow.arr(name)), name
    for p, q in zip(w.collPts, ow.coll_pts()):
        assert (p.body, p.lx, p.ly, p.r) == q
    oc = ow.constraints
    for c, d in zip(w.constraints, oc):
        for f in ("type", "a", "b", "lax", "lay", "lbx", "lby", "compliance", "broken",
                  "breakForce", "target", "rest", "minAngle", "maxAngle", "owner", "color"):
            assert getattr(c, f) == getattr(d, f), f
    off, cnt = ow.color_info()
    assert list(w.colorOff) == off and list(w.colorCnt) == cnt


def test_apply_control_and_proprio_match():
    sim = core.create_sim(seed=23, creatures=1)
    c = sim["creatures"][0]
    o = ob.Sim(seed=23, creatures=1)
    rnd = world_map.mulberry32(4)
    for i in range(5):
        tone = rnd()
        sh = [rnd() * 2 - 1 for _ in range(6)]
        cu = [rnd() * 2 - 1 for _ in range(6)]
        ad = [rnd() for _ in range(6)]
        core.apply_control(c, {"tone": tone, "arms": [{"shoulder": sh[a], "curl": cu[a],
                                                       "adhesion": ad[a]} for a in range(6)]})
        o.apply_control(0, tone, sh, cu, ad)
        p1 = core.read_proprio(c)
        p2 = o.read_proprio(0)
        assert np.array_equal(p1, p2)
    for a, d in zip(sim["world"].constraints, o.world.constraints):
        assert (a.target, a.compliance, a.broken, a.breakForce, a.lbx, a.lby) == \
               (d.target, d.compliance, d.broken, d.breakForce, d.lbx, d.lby)


def test_ensure_colored_regroups_creation_order():
    # gpu.html buildWorld worlds are uncoloured; create() colours them
    w = xpbd.XpbdWorld()
    kraken.spawn_kraken(w, 700, 400, 0.3)
    ow = ob.World()
    ow.spawn_kraken(700, 400, 0.3)
    xpbd.ensure_colored(w)
    ow.ensure_colored()
    ids = ow.list_ids()
    for c, i in zip(w.constraints, ids):
        d = ow.con(int(i))
        assert (c.type, c.a, c.b, c.color) == (d.type, d.a, d.b, d.color)
    assert list(w.colorCnt) == ow.color_info()[1]


def test_colour_mask_overflow_matches_typed_array_semantics():
    # createSim's mask has 1 << 16 entries (core.js:45); 1526 creatures put
    # bodies past its end, where the Uint32Array reads 0 and drops writes
    n = 1526
    sim = core.create_sim(seed=2, creatures=n)
    o = ob.Sim(seed=2, creatures=n)
    assert sim["world"].n > 1 << 16
    off, cnt = o.world.color_info()
    assert list(sim["world"].colorCnt) == cnt
    ids = o.world.list_ids()
    tail = slice(len(ids) - 500, len(ids))
    for c, i in zip(sim["world"].constraints[tail], ids[tail]):
        d = o.world.con(int(i))
        assert (c.a, c.b, c.color) == (d.a, d.b, d.color)
