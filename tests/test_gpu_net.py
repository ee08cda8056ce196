"""KR_CTRL_NET on the device against the oracle's trainStep (src/sim/
train.js:233-249): the reference net (src/brain/net.js) on proprioception,
senses (echo, light, contact; no entities) and its own previous outputs,
driving the f32 XPBD step, creature by creature over uneven bodies and maps.

Physics and the f32 data path are bit-exact; the f64 libm calls (tanh,
sin, cos, atan2, hypot) of the controller may differ from glibc in the last
f64 bit, which would move an f32 rounding of an input or output by one ulp
and then grow through the closed loop.  Measured: every creature of the
60-step scenario bit-identical to the oracle at every step; the tests allow
one creature with such a rounding, bounded by the f64 tolerance class."""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, workloads
from tests.test_net_host import _net_sim, random_genome

pytestmark = pytest.mark.gpu


def _genomes(w, seed, echo_bias=None):
    rng = np.random.default_rng(seed)
    G = []
    for i in range(w.n):
        A = int(w.arms[i])
        g = random_genome(batch.net_inputs(A), batch.net_outputs(A), rng)
        if echo_bias is not None:
            g[-1] = echo_bias
        G.append(g)
    return G


def _run_net(w, G, steps, lanes=None):
    """The engine over all creatures; genomes of several arm counts padded
    to one row width."""
    eng = batch.BatchEngine(w.maps, w.n, control="net", lights=w.lights)
    workloads.spawn_all(eng, w)
    if lanes:
        eng.set_launch(4, 0, lanes_per_creature=lanes)
    width = max(len(g) for g in G)
    padded = np.zeros((len(G), width), np.float32)
    for k, g in enumerate(G):
        padded[k, :len(g)] = g
    eng.set_net(padded, np.arange(w.n, dtype=np.int32))
    eng.run(steps)
    x, o = eng.read_net()
    metrics = eng.read_metrics()
    eng.close()
    return x, o, metrics


def test_net_first_step():
    """Step 1 (zero senses and outputs in, the spawn pose): inputs and
    outputs within 1e-6 (the proprioception's f64 libm), nearly all exact."""
    w = workloads.uneven(n=8, n_maps=2, seed=23, h_min=1, h_max=1, arms=(5, 5), segs=(5, 9))
    G = _genomes(w, 4)
    x, o, _ = _run_net(w, G, 1)
    exact = total = 0
    for i in range(w.n):
        sim, net, hist = _net_sim(w, i, 1, G[i])
        xi, oi = hist[-1]
        A = int(w.arms[i])
        ni, no = batch.net_inputs(A), batch.net_outputs(A)
        assert np.allclose(x[i, :ni], xi, atol=1e-6, rtol=0) and np.allclose(o[i, :no], oi, atol=1e-6, rtol=0)
        exact += int(np.sum(x[i, :ni] == xi)) + int(np.sum(o[i, :no] == oi))
        total += ni + no
    assert exact >= 0.98 * total, (exact, total)


@pytest.mark.parametrize("lanes", [32, 16, 8])
def test_net_engine_matches_oracle_trainer(lanes):
    """60 trainer steps per creature, every step's input vector and outputs
    compared: bit-identical for (nearly) every creature; a creature whose
    f64 libm call rounded differently once stays within 1e-4 for the first
    10 steps and within 0.05 px of the oracle's mantle after 60."""
    w = workloads.uneven(n=12, n_maps=3, seed=21, h_min=60, h_max=60, arms=(6, 6), segs=(5, 9))
    G = _genomes(w, 3, echo_bias=1.5)
    eng = batch.BatchEngine(w.maps, w.n, control="net", lights=w.lights)
    workloads.spawn_all(eng, w)
    eng.set_launch(4, 0, lanes_per_creature=lanes)
    eng.set_net(np.stack(G), np.arange(w.n, dtype=np.int32))
    X, O = [], []
    for t in range(60):
        eng.run(1)
        x, o = eng.read_net()
        X.append(x.copy())
        O.append(o.copy())
    metrics = eng.read_metrics()
    eng.close()
    identical = 0
    for i in range(w.n):
        sim, net, hist = _net_sim(w, i, 60, G[i])
        ni, no = batch.net_inputs(6), batch.net_outputs(6)
        same = all(np.array_equal(X[t][i, :ni], hist[t][0]) and np.array_equal(O[t][i, :no], hist[t][1])
                   for t in range(60))
        identical += same
        want = sim.metrics(0)
        got = dict(zip(batch.METRIC_FIELDS, metrics[i]))
        if same:
            for f in ("x", "y", "pathLen", "energySpent", "gripCycles", "attachEvents"):
                assert np.isclose(got[f], want[f], rtol=1e-10, atol=1e-9), (i, f, got[f], want[f])
        else:
            for t in range(10):
                assert np.allclose(X[t][i, :ni], hist[t][0], atol=1e-4, rtol=0), (i, t)
            assert abs(got["x"] - want["x"]) < 0.05 and abs(got["y"] - want["y"]) < 0.05, i
        assert got["steps"] == 60
    assert identical >= w.n - 1, identical
    P, E = 6 * 6 + 6, 2 * batch.NET_RAYS
    assert np.any(X[-1][:, P:P + E] > 0)                              # echoes arrived
    assert np.any(X[-1][:, P + E + 6:P + E + 9] > np.float32(0.05))   # lit somewhere


def test_net_same_for_every_launch_shape_and_alone():
    """A creature's net rollout does not depend on the launch shape, its
    neighbours (of other arm counts too) or its slot."""
    w = workloads.uneven(n=16, n_maps=3, seed=25, h_min=80, h_max=80, arms=(4, 8), segs=(5, 9))
    G = _genomes(w, 6, echo_bias=1.0)
    x, o, metrics = _run_net(w, G, 80, lanes=8)
    for lanes in (16, 32):
        x2, o2, m2 = _run_net(w, G, 80, lanes=lanes)
        assert np.array_equal(x2, x) and np.array_equal(o2, o) and np.array_equal(m2, metrics)
    for i in (0, 7, 15):
        sub = workloads.Workload("one", w.maps, w.arms[i:i + 1], w.segs[i:i + 1], w.map_id[i:i + 1],
                                 w.x[i:i + 1], w.y[i:i + 1], w.angle[i:i + 1], w.horizon[i:i + 1],
                                 w.seed[i:i + 1], w.lights)
        x1, o1, m1 = _run_net(sub, [G[i]], 80)
        assert np.array_equal(x1[0], x[i]) and np.array_equal(o1[0], o[i])
        assert np.array_equal(m1[0], metrics[i])


def test_server_net_request_equals_engine_with_host_perturbed_genomes():
    """A mirrored ES request under the reference net: the server perturbs the
    genome on the device into the net's device layout; the engine given the
    same theta +- sigma * eps (eps from the device generator, f32 arithmetic
    on the host) in net.js's own layout gives the same bits."""
    from kraken_3_gpu_b200 import serve
    w = workloads.uneven(n=4, n_maps=3, seed=31, h_min=10, h_max=10)
    arms, segs, pop, H, m = 6, 7, 6, 70, 1
    x, y = float(w.x[0]), float(w.y[0])
    m = int(w.map_id[0])
    rng = np.random.default_rng(8)
    n_par = batch.net_param_count(arms)
    theta = random_genome(batch.net_inputs(arms), batch.net_outputs(arms), rng)
    theta[-1] = 1.0  # the echo fires
    sigma, seed = 0.05, 123
    srv = serve.Server(w.maps, 1 << 30, max_slots=32, chunk_steps=16, net=True, lights=w.lights)
    rid = srv.submit(pop, H, arms, segs, m, x, y, 0.4, theta=theta, sigma=sigma, seed=seed)
    srv.drain()
    got = srv.result(rid, pop)["results"]
    srv.close()
    G = []
    for i in range(pop):
        d = np.float32(sigma) * serve.policy_eps(seed, i // 2, n_par)
        G.append(theta + d if i % 2 == 0 else theta - d)
    eng = batch.BatchEngine(w.maps, pop, control="net", lights=w.lights)
    eng.spawn(0, [arms] * pop, [segs] * pop, [m] * pop, [x] * pop, [y] * pop, [0.4] * pop, [H] * pop)
    eng.set_net(np.stack(G), np.arange(pop, dtype=np.int32))
    eng.run(H)
    want = eng.read_metrics()
    eng.close()
    assert np.array_equal(got, want)
    assert not np.array_equal(got[0], got[1])  # the mirrored pair differs


def test_net_restore_and_autotune_keep_the_sense_state():
    """The net record (echo queue, lights, contact, recurrent outputs) is part
    of a slot's state: a rollout restored from a snapshot repeats itself, and
    the autotuner's trial launches leave the slots as they were."""
    w = workloads.uneven(n=16, n_maps=2, seed=27, h_min=90, h_max=90, arms=(6, 6), segs=(5, 9))
    G = _genomes(w, 9, echo_bias=1.5)
    eng = batch.BatchEngine(w.maps, w.n, control="net", lights=w.lights)
    workloads.spawn_all(eng, w)
    eng.set_net(np.stack(G), np.arange(w.n, dtype=np.int32))
    eng.run(30)
    eng.snapshot()
    eng.run(60)
    first = (eng.read_net(), eng.read_metrics())
    eng.restore()
    eng.autotune(8)
    eng.run(60)
    second = (eng.read_net(), eng.read_metrics())
    eng.close()
    assert np.array_equal(first[0][0], second[0][0]) and np.array_equal(first[0][1], second[0][1])
    assert np.array_equal(first[1], second[1])


def _host_light_sense(lights, steps, dt, x, y, ang0, mw=1440.0, mh=810.0):
    """light.js sampleAt for the three receptors after `steps` ticks of the
    map's lights (map.js tickMapLights), in numpy f64 from the map's initial
    positions; (x, y, ang0) the creature's mantle."""
    L = np.asarray(lights, np.float64).reshape(-1, 6)
    px, py = L[:, 0].copy(), L[:, 1].copy()
    time = 0.0
    for _ in range(steps):
        time = time + dt
        a = time * L[:, 5] + L[:, 4]
        px = np.maximum(60.0, np.minimum(mw - 60, px + np.cos(a) * 18 * dt))
        py = np.maximum(60.0, np.minimum(mh - 60, py + np.sin(a * 0.8) * 18 * dt))
    heading = float(ang0) - np.pi * 0.5
    sp, cp = np.sin(heading + np.pi / 2), np.cos(heading + np.pi / 2)
    pts = [(x + cp * 26, y + sp * 26), (x - cp * 26, y - sp * 26), (x, y)]
    out = []
    for qx, qy in pts:
        v = 0.05
        for k in range(len(L)):
            d = np.hypot(qx - px[k], qy - py[k])
            v += max(0.0, 1 - d / L[k, 2]) * L[k, 3]
        out.append(min(1.0, v))
    return np.asarray(out, np.float32)


@pytest.mark.parametrize("steps", [100, 4200])
def test_light_sense_from_the_table_and_past_it(steps):
    """The lights' positions come from the engine's per-map table for the
    first 4,096 env steps (every creature of a map sees the same lights after
    its step t) and are ticked per creature after it.  The light inputs of
    the last step, built from the senses at the end of the step before,
    against the lights ticked on the host for as many steps and the
    creature's pose then: within 1e-6 (libm cos / sin / hypot may differ in
    the last f64 bit), before and after the end of the table."""
    w = workloads.uneven(n=4, n_maps=2, seed=31, h_min=steps, h_max=steps, arms=(5, 5), segs=(5, 5))
    G = _genomes(w, 6)
    eng = batch.BatchEngine(w.maps, w.n, control="net", lights=w.lights)
    workloads.spawn_all(eng, w)
    width = max(len(g) for g in G)
    padded = np.zeros((len(G), width), np.float32)
    for k, g in enumerate(G):
        padded[k, :len(g)] = g
    eng.set_net(padded, np.arange(w.n, dtype=np.int32))
    eng.run(steps - 1)
    st = eng.read_state()
    eng.run(1)
    x, _ = eng.read_net()
    eng.close()
    dt = (1 / 120) * 2
    for i in range(w.n):
        A = int(w.arms[i])
        at = 6 * A + 6 + 2 * batch.NET_RAYS + 6  # proprioception, echo, chemoreception, then light
        want = _host_light_sense(w.lights[w.map_id[i]], steps - 1, dt, float(st["px"][i, 0]),
                                 float(st["py"][i, 0]), st["ang"][i, 0])
        assert np.allclose(x[i, at:at + 3], want, atol=1e-6, rtol=0), (i, x[i, at:at + 3], want)
