"""The reference trainer's controller on the host: the oracle's forwardInto
against a line-by-line Python restatement of src/brain/net.js:71-98 (same
libm, so bit-identical), the lights of makeMap (src/world/map.js:60-69), and
the oracle's trainStep invariants (input layout of core.js:113-122 and
:226-232, echo bookkeeping of src/senses/echo.js)."""
import math

import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, kraken, workloads
from kraken_3_gpu_b200.world_map import light_array, make_map
from oracle import binding as ob


def random_genome(n_in, n_out, rng, hidden=24):
    """randomGenome (net.js:41-55): N(0, 1/fan_in) weights -- here with
    nonzero biases too, so that every weight block is exercised."""
    w = np.zeros(batch.net_param_count((n_in - 45) // 10), np.float32)
    i = 0
    for n, s in ((n_in * hidden, 1 / math.sqrt(n_in)), (hidden, 0.3), (hidden * hidden, 1 / math.sqrt(hidden)),
                 (hidden, 0.3), (hidden * n_out, 1 / math.sqrt(hidden)), (n_out, 0.3)):
        w[i:i + n] = rng.normal(0, s, n)
        i += n
    assert i == len(w) and n_out == 3 * ((n_in - 45) // 10) + 2
    return w


def forward_py(w, x, n_out, hidden=24):
    n_in = len(x)
    b1 = n_in * hidden
    b2 = b1 + hidden
    b3 = b2 + hidden * hidden
    b4 = b3 + hidden
    b5 = b4 + hidden * n_out
    act = lambda s: 1.0 if s > 20 else (-1.0 if s < -20 else math.tanh(s))
    h1 = np.zeros(hidden, np.float32)
    h2 = np.zeros(hidden, np.float32)
    out = np.zeros(n_out, np.float32)
    for j in range(hidden):
        s = float(w[b1 + j])
        for i in range(n_in):
            s += float(x[i]) * float(w[j * n_in + i])
        h1[j] = act(s)
    for j in range(hidden):
        s = float(w[b2 + j])
        row = b3 - hidden * hidden + j * hidden
        for i in range(hidden):
            s += float(h1[i]) * float(w[row + i])
        h2[j] = act(s)
    for j in range(n_out):
        s = float(w[b5 + j])
        for i in range(hidden):
            s += float(h2[i]) * float(w[b4 + j * hidden + i])
        out[j] = act(s)
    return out


@pytest.mark.parametrize("arms", [6, 4, 8])
def test_oracle_forward_equals_python_restatement(arms):
    rng = np.random.default_rng(arms)
    n_in, n_out = batch.net_inputs(arms), batch.net_outputs(arms)
    assert ob.net_param_count(arms) == batch.net_param_count(arms)
    for _ in range(3):
        w = random_genome(n_in, n_out, rng)
        x = rng.uniform(-1.2, 1.2, n_in).astype(np.float32)
        assert np.array_equal(ob.net_forward(w, x, n_out), forward_py(w, x, n_out))
    # saturation beyond +-20 and the bias of the second layer read at b2 + j
    w = np.zeros(batch.net_param_count(arms), np.float32)
    w[n_in * 24:n_in * 24 + 24] = 30.0           # first-layer bias: h1 = 1
    w[n_in * 24 + 24] = 0.25                     # W2 row 0, col 0 == the bias of h2[0]
    out = ob.net_forward(w, np.zeros(n_in, np.float32), n_out)
    assert np.array_equal(out, forward_py(w, np.zeros(n_in, np.float32), n_out))


def test_reference_net_size():
    assert batch.net_param_count(6) == 3644  # net.js: 105 -> 24 -> 24 -> 20
    assert batch.net_inputs(6) == 105 and batch.net_outputs(6) == 20


def test_make_map_lights():
    m = make_map(1440, 810, seed=1)
    L = np.array(light_array(m))
    assert L.shape == (4, 6)
    assert np.all((L[:, 0] >= 14) & (L[:, 0] <= 1440 - 14) & (L[:, 1] >= 14) & (L[:, 1] <= 810 - 14))
    assert np.all((L[:, 2] >= 220) & (L[:, 2] < 290) & (L[:, 3] >= 0.7) & (L[:, 3] < 0.82))
    assert np.all((L[:, 4] >= 0) & (L[:, 4] < 2 * math.pi) & (L[:, 5] >= 0.11) & (L[:, 5] < 0.17))
    # drawn after the rects from the same stream: the rects do not change
    assert make_map(1440, 810, seed=1, lights=0)["rects"] == m["rects"]
    assert len(make_map(1440, 810, seed=3, lights=7)["lights"]) == 7


def _net_sim(w, i, steps, genome):
    rects = w.maps[w.map_id[i]].astype(np.float32).astype(np.float64)
    sim = ob.Sim(rects=rects)
    sim.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
    sim.world.f32ify()
    sim.world.round_state()
    sim.set_spawn_reach(0, ob.measure_reach(rects, kraken.arm_reach(int(w.segs[i])), w.x[i], w.y[i]))
    net = ob.NetSim(sim, w.lights[w.map_id[i]])
    hist = []
    for _ in range(steps):
        net.step(genome[None], [0])
        hist.append(net.io(0))
    return sim, net, hist


def test_oracle_trainer_step_input_layout_and_echo():
    w = workloads.uneven(n=6, n_maps=2, seed=11, h_min=120, h_max=120)
    rng = np.random.default_rng(5)
    emitted = 0
    for i in range(w.n):
        A = int(w.arms[i])
        g = random_genome(batch.net_inputs(A), batch.net_outputs(A), rng)
        g[-1] = 2.0  # echo output biased on: the echo fires whenever the cooldown allows
        sim, net, hist = _net_sim(w, i, 120, g)
        P, E = 6 * A + 6, 2 * batch.NET_RAYS
        for t, (x, out) in enumerate(hist):
            assert np.all(x[P + E:P + E + 6] == 0) and np.all(x[P + E + 9:P + E + 13] == 0)  # chem, hearing
            light = x[P + E + 6:P + E + 9]
            assert np.all((light >= np.float32(0.05)) | (t == 0)) and np.all(light <= 1)
            contact = x[P + E + 13:P + E + 13 + A]
            assert np.all((contact >= 0) & (contact <= 1))
            prev = hist[t - 1][1] if t else np.zeros_like(out)
            assert np.array_equal(x[P + E + 13 + A:], prev)        # recurrent inputs
            assert np.all(np.abs(out) <= 1)
        emits, pending = net.echo(0)
        # one emission per 26 steps (0.42 s at 1/60 s) at most, <= 2 emissions pending
        assert 1 <= emits <= 120 // 26 + 1 and pending <= 2 * batch.NET_RAYS
        emitted += emits
        echo = hist[-1][0][P:P + E]
        assert np.all((echo >= 0) & (echo <= 1))
    assert emitted > 0


def test_net_engine_rejects_bad_light_descriptors():
    """Host validation runs before any device work: too many lights on a map,
    a light without a positive radius."""
    w = workloads.uneven(n=2, n_maps=1, seed=1)
    lights = [np.zeros((batch.NET_MAX_LIGHTS + 1, 6)) + [100, 100, 250, 0.7, 0, 0.1]]
    with pytest.raises(Exception, match="lights"):
        batch.BatchEngine(w.maps, 2, control="net", lights=lights)
    with pytest.raises(Exception, match="radius"):
        batch.BatchEngine(w.maps, 2, control="net", lights=[[[100, 100, 0, 0.7, 0, 0.1]]])
