"""Generates the golden fixtures of tests/golden from the oracle.

    python tests/golden/make_golden.py

The reference keeps no stored per-particle vectors (its checks are property
checks and quoted results), so these fixtures are the oracle's own outputs on
seeded scenarios, committed to pin the oracle against drift and to give the
GPU tests fixed expected values:

config0.npz  the single-creature scenario: createSim(seed 1, 1 creature) on
             map seed 1, tone 0.5, 42 muscle targets ~ U[-1, 1] and 6
             adhesion values ~ U[0, 1] redrawn every 6 steps from
             mulberry32(0) (draw order per arm: motors, then adhesion), run by
             the FP64 oracle (xpbd.js) and the f32 oracle (f32solver.mjs); the
             body state after steps 1, 10 and 60 and the grip flags of every
             arm before and after every step.
batch.npz    eight creatures of the mixed workload (workloads.uneven(n=8,
             n_maps=2, seed=5, horizons 30)) each run alone by the f32 oracle
             with its control stream for 30 steps: body state and grip flags.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FIELDS = ("px", "py", "vx", "vy", "ang", "av")
CHECKPOINTS = (1, 10, 60)


def config0(f32: bool):
    from kraken_3_gpu_b200.workloads import TONE, ControlStream
    from oracle import binding as ob
    o = ob.Sim(seed=1, creatures=1)
    if f32:
        o.world.f32ify()
        o.world.round_state()
    cs = ControlStream(seed=0)
    oc = o.creatures[0]
    out = {}
    grips = []
    for s in range(max(CHECKPOINTS)):
        t, a = cs.at(s)
        o.apply_control_motors(0, TONE, t, a)
        before = [oc.grip(k).broken for k in range(6)]
        (o.step32 if f32 else o.step)()
        after = [oc.grip(k).broken for k in range(6)]
        grips.append([before, after])
        if s + 1 in CHECKPOINTS:
            for f in FIELDS:
                out[f"{f}_{s + 1}"] = o.world.arr(f).astype(np.float32 if f32 else np.float64)
    out["grips"] = np.array(grips, dtype=np.uint8)
    return out


def batch():
    from kraken_3_gpu_b200 import workloads
    from kraken_3_gpu_b200.workloads import TONE, ControlStream
    from oracle import binding as ob
    w = workloads.uneven(n=8, n_maps=2, seed=5, h_min=30, h_max=30)
    nbm = 1 + 8 * 9
    out = {f: np.zeros((w.n, nbm), np.float32) for f in FIELDS}
    out["grips"] = np.zeros((w.n, 8), np.uint8)
    for i in range(w.n):
        sim = ob.Sim(rects=w.maps[w.map_id[i]])
        k = sim.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
        sim.world.f32ify()
        sim.world.round_state()
        cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
        for s in range(30):
            t, a = cs.at(s)
            sim.apply_control_motors(0, TONE, t, a)
            sim.step32()
        nb = sim.world.n
        for f in FIELDS:
            out[f][i, :nb] = sim.world.arr(f).astype(np.float32)
        for a in range(int(w.arms[i])):
            out["grips"][i, a] = 1 if k.grip(a).broken else 0
    return out


def main():
    np.savez_compressed(os.path.join(HERE, "config0_f64.npz"), **config0(False))
    np.savez_compressed(os.path.join(HERE, "config0_f32.npz"), **config0(True))
    np.savez_compressed(os.path.join(HERE, "batch_f32.npz"), **batch())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")


if __name__ == "__main__":
    main()
