"""GPU parity of the batched engine (uneven bodies, several maps, device
reflex and proprioception) against the f32 oracle, creature by creature.

Each creature of the batch must equal a one-creature f32-oracle world on its
map at its spawn pose, driven by the reference's hybrid loop with the same
control stream: bit-identical body state and grip flags (the engine runs the
same f32 op sequence; reflex and proprioception are f64 on both sides), and
proprioception within 1e-6 of the oracle's readProprio.
"""
import numpy as np
import pytest

from kraken_3_gpu_b200 import batch, workloads
from oracle import binding as ob
from tests.scenarios import TONE, ControlStream

pytestmark = pytest.mark.gpu


def _small_uneven(n=24, n_maps=4, h=40):
    w = workloads.uneven(n=n, n_maps=n_maps, seed=5, h_min=h, h_max=h)
    return w


def _oracle_run(w, i, steps, record_obs=False):
    sim = ob.Sim(rects=w.maps[w.map_id[i]])
    k = sim.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
    sim.world.f32ify()
    sim.world.round_state()
    cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
    obs = []
    for s in range(steps):
        if record_obs:
            obs.append(sim.read_proprio(0))
        t, a = cs.at(s)
        # the engine's stream draws into its f32 control record
        t32, a32 = (v.astype(np.float32).astype(np.float64) for v in (t, a))
        sim.apply_control_motors(0, TONE, t32, a32)
        sim.step32()
    grips = [k.grip(a).broken for a in range(int(w.arms[i]))]
    return sim, grips, obs


def test_uneven_batch_bit_exact_vs_f32_oracle():
    w = _small_uneven()
    eng = batch.BatchEngine(w.maps, w.n, obs_ring=64)
    workloads.spawn_all(eng, w)
    eng.run(40)
    st = eng.read_state()
    obs = eng.read_obs()
    assert np.all(st["steps"] == 40)
    exact = total = 0
    for i in range(w.n):
        sim, grips, o_obs = _oracle_run(w, i, 40, record_obs=True)
        nb = sim.world.n
        for f in ("px", "py", "ang", "vx", "vy", "av"):
            got = st[f][i, :nb]
            ref = sim.world.arr(f).astype(np.float32)
            assert np.array_equal(got, ref), f"creature {i} ({w.arms[i]}x{w.segs[i]}) field {f}"
        assert [bool(g) for g in st["grips"][i, : int(w.arms[i]), 3]] == grips
        A = int(w.arms[i])
        for s in range(40):
            p = obs[i, s, : 6 * A + 6]
            assert np.allclose(p, o_obs[s], atol=1e-6, rtol=0), (i, s)
            exact += int(np.sum(p == o_obs[s].astype(np.float32)))
            total += 6 * A + 6
            flags = int(obs[i, s, batch.OBS_STRIDE - 1].view(np.uint32))
            assert flags == sum(1 << a for a in range(A) if o_obs[s][5 * A + a] == 1.0)
    # the f64 libm (atan2, sin, cos, hypot) may move an f32 rounding by one ulp
    # now and then; everything else is the oracle's value bit for bit
    assert exact >= 0.999 * total, (exact, total)
    eng.close()


def test_chunked_runs_and_graph_equal_one_run():
    w = _small_uneven(n=16, h=60)
    ref = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(ref, w)
    ref.run(60)
    a = ref.read_state()
    chunked = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(chunked, w)
    for _ in range(6):
        chunked.run(10)
    b = chunked.read_state()
    graphed = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(graphed, w)
    graphed.run_graph(15, launches=4, replays=1)
    c = graphed.read_state()
    for f in ("px", "py", "ang", "vx", "vy", "av"):
        assert np.array_equal(a[f], b[f]) and np.array_equal(a[f], c[f]), f
    assert np.all(a["steps"] == 60) and np.all(c["steps"] == 60)
    for e in (ref, chunked, graphed):
        e.close()


@pytest.mark.parametrize("slice_ms", [0.3, 2.0])
def test_time_sliced_run_equals_one_launch(slice_ms):
    """Preemptible time slices (creatures stopped mid-rollout, regrouped and
    relaunched) end in the one launch's state and metrics, bit for bit; a
    step-limited run (max_steps short of the horizons) stays one launch."""
    w = workloads.uneven(n=700, n_maps=6, seed=21, h_min=40, h_max=900)
    H = int(w.horizon.max())
    ref = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(ref, w)
    ref.run(H)
    a, ma = ref.read_state(), ref.read_metrics()
    ref.close()
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.set_slice(slice_ms)
    eng.set_launch(8, 0, lanes_per_creature=16)
    eng.run(H // 3)
    assert eng.last_run_launches() == (1, 1, w.n)
    eng.set_launch(0, 0, lanes_per_creature=0)  # the automatic shape of every slice
    live = int(np.sum(w.horizon > H // 3))
    eng.run(H)
    slices, kernels, launched = eng.last_run_launches()
    assert slices > 1 and kernels in (2 * slices - 1, 2 * slices) and launched >= live + slices - 1
    assert eng.last_ms() > 0
    b, mb = eng.read_state(), eng.read_metrics()
    eng.close()
    for f in ("px", "py", "ang", "vx", "vy", "av", "steps"):
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(ma, mb)
    assert np.array_equal(b["steps"], w.horizon)


@pytest.mark.parametrize("lanes,warps,ctas,unroll", [(32, 1, 1, 1), (32, 16, 1, 2), (16, 4, 2, 1), (16, 8, 0, 2),
                                                      (8, 2, 4, 1), (8, 16, 1, 1), (8, 8, 0, 2), (16, 4, 5, 1),
                                                      (16, 4, 6, 2), (32, 8, 3, 1)])
def test_launch_shape_does_not_change_results(lanes, warps, ctas, unroll):
    """One to four creatures per warp, any CTA size or CTAs per SM, the
    substep loop rolled or unrolled: the same bits."""
    w = _small_uneven(n=40, h=30)
    base = batch.BatchEngine(w.maps, w.n, obs_ring=32)
    workloads.spawn_all(base, w)
    base.run(30)
    other = batch.BatchEngine(w.maps, w.n, obs_ring=32)
    other.set_launch(warps, ctas, lanes_per_creature=lanes)
    other.set_unroll(unroll)
    workloads.spawn_all(other, w)
    other.run(17)
    other.run(13)
    assert other.get_launch()["lanes_per_creature"] == lanes
    assert other.get_launch()["substep_unroll"] == unroll
    s0, s1 = base.read_state(), other.read_state()
    for f in ("px", "py", "ang", "vx", "vy", "av", "grips", "steps"):
        assert np.array_equal(s0[f], s1[f]), f
    assert np.array_equal(base.read_obs(), other.read_obs())
    assert np.array_equal(base.read_metrics(), other.read_metrics())
    base.close()
    other.close()


def test_horizons_stop_each_creature():
    w = workloads.uneven(n=12, n_maps=2, seed=9, h_min=5, h_max=25)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(100)
    st = eng.read_state()
    assert np.array_equal(st["steps"], w.horizon)
    assert eng.live() == 0
    eng.close()


def _mlp_reference(w, obs, arms, segs):
    """The fused controller in f64: proprio -> 64 tanh -> A*S tanh targets
    and A (tanh + 1) / 2 adhesion values (kraken_batch.h layout)."""
    n_in, n_out, H = 6 * arms + 6, arms * segs + arms, batch.POLICY_HIDDEN
    W1 = w[: H * (n_in + 1)].reshape(H, n_in + 1).astype(np.float64)
    W2 = w[H * (n_in + 1): H * (n_in + 1) + n_out * (H + 1)].reshape(n_out, H + 1).astype(np.float64)
    h = np.tanh(W1[:, :n_in] @ obs[:n_in].astype(np.float64) + W1[:, n_in])
    y = np.tanh(W2[:, :H] @ h + W2[:, H])
    y[arms * segs:] = 0.5 * (y[arms * segs:] + 1.0)
    return y


@pytest.mark.parametrize("lanes", [32, 16, 8])
def test_fused_policy_matches_mlp_on_recorded_proprio(lanes):
    w = _small_uneven(n=12, h=6)
    rng = np.random.default_rng(3)
    n_params = batch.policy_params(8, 9)
    n_ind = w.n  # one individual per creature (weights are laid out per body shape)
    weights = rng.normal(0.0, 0.3, size=(n_ind, n_params)).astype(np.float32)
    slot_ind = rng.permutation(n_ind).astype(np.int32)
    eng = batch.BatchEngine(w.maps, w.n, obs_ring=8, control="policy")
    eng.set_launch(4, 0, lanes_per_creature=lanes)
    workloads.spawn_all(eng, w)
    eng.set_policy(weights, slot_ind)
    for step in range(3):
        eng.run(1)
        obs = eng.read_obs()
        ctrl = eng.read_controls()
        for i in range(w.n):
            A, S = int(w.arms[i]), int(w.segs[i])
            want = _mlp_reference(weights[slot_ind[i]], obs[i, step], A, S)
            got = ctrl[i, : A * S + A]
            assert np.allclose(got, want, atol=2e-5, rtol=0), (i, step)
    eng.close()


def test_fused_policy_same_bits_for_every_launch_shape():
    w = _small_uneven(n=20, h=25)
    rng = np.random.default_rng(4)
    weights = rng.normal(0.0, 0.2, size=(w.n, batch.policy_params(8, 9))).astype(np.float32)
    slot_ind = rng.permutation(w.n).astype(np.int32)
    out = []
    for lanes, warps in ((32, 8), (16, 4), (8, 16)):
        eng = batch.BatchEngine(w.maps, w.n, control="policy")
        eng.set_launch(warps, 0, lanes_per_creature=lanes)
        workloads.spawn_all(eng, w)
        eng.set_policy(weights, slot_ind)
        eng.run(25)
        out.append(eng.read_state())
        eng.close()
    for s in out[1:]:
        for f in ("px", "py", "ang", "grips"):
            assert np.array_equal(out[0][f], s[f]), f


def test_policy_individual_shared_by_two_body_shapes_is_rejected():
    from kraken_3_gpu_b200 import _native
    w = _small_uneven(n=12, h=6)
    assert len(set(zip(w.arms.tolist(), w.segs.tolist()))) > 1
    eng = batch.BatchEngine(w.maps, w.n, control="policy")
    workloads.spawn_all(eng, w)
    weights = np.zeros((1, batch.policy_params(8, 9)), np.float32)
    with pytest.raises(_native.KrError) as e:
        eng.set_policy(weights, np.zeros(w.n, np.int32))
    assert "two body shapes" in str(e.value)
    eng.close()


def test_autotune_leaves_slots_as_they_were():
    w = _small_uneven(n=48, h=40)
    ref = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(ref, w)
    ref.run(15)
    ref.run(25)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.run(15)
    before = eng.read_state()
    lanes, warps, ctas, ms = eng.autotune(10)
    assert lanes in (8, 16, 32) and ms > 0
    assert eng.get_launch()["lanes_per_creature"] == lanes
    after = eng.read_state()
    for f in ("px", "py", "ang", "vx", "vy", "av", "grips", "steps"):
        assert np.array_equal(before[f], after[f]), f
    eng.run(25)
    a, b = ref.read_state(), eng.read_state()
    for f in ("px", "py", "ang", "grips", "steps"):
        assert np.array_equal(a[f], b[f]), f
    assert np.array_equal(ref.read_metrics(), eng.read_metrics())
    ref.close()
    eng.close()


@pytest.mark.parametrize("lanes", [8, 16, 32])
def test_creatures_against_walls_bit_exact_vs_f32_oracle(lanes):
    """Creatures spawned with their arms across the walls of their map, so
    that collision passes correct many points every step (the culled list,
    the per-body skip and the sequential commit all active): body state equal
    to the f32 oracle bit for bit after 30 steps, under every lane count."""
    w = _small_uneven(n=12, n_maps=3, h=30)
    rng = np.random.default_rng(17)
    for i in range(w.n):
        r = w.maps[w.map_id[i]]
        # an inner wall where the map has one (the first four rects are the border)
        k = 4 + int(rng.integers(0, len(r) - 4)) if len(r) > 4 else int(rng.integers(0, 4))
        x, y, rw, rh = (float(v) for v in r[k])
        reach = 24 + 13.5 * int(w.segs[i])
        if rw < rh:   # vertical wall: mantle beside it on the map's side, arms across it
            w.x[i] = x - 0.6 * reach if x > 720 else x + rw + 0.6 * reach
            w.y[i] = y + 0.5 * rh
        else:
            w.x[i] = x + 0.5 * rw
            w.y[i] = y - 0.6 * reach if y > 405 else y + rh + 0.6 * reach
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.set_launch(4 if lanes == 32 else 8, 0, lanes_per_creature=lanes)
    eng.run(30)
    st = eng.read_state()
    eng.close()
    moved_by_walls = 0
    for i in range(w.n):
        sim, grips, _ = _oracle_run(w, i, 30)
        nb = sim.world.n
        for f in ("px", "py", "ang", "vx", "vy", "av"):
            assert np.array_equal(st[f][i, :nb], sim.world.arr(f).astype(np.float32)), (i, f)
        free = ob.Sim(rects=np.zeros((0, 4)))  # the same creature with no map: how far walls moved it
        free.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
        free.world.f32ify()
        free.world.round_state()
        cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
        for s in range(30):
            t, a = cs.at(s)
            t32, a32 = (v.astype(np.float32).astype(np.float64) for v in (t, a))
            free.apply_control_motors(0, TONE, t32, a32)
            free.step32()
        moved_by_walls += not np.array_equal(free.world.arr("px"), sim.world.arr("px"))
    assert moved_by_walls >= w.n // 2, moved_by_walls  # the walls acted on most creatures


def test_device_sincos_is_the_rounded_f64_value():
    """The solver's f64 sin / cos rounded to f32 against numpy's f64 sin / cos
    rounded to f32, on 2 M angles up to 2^20 rad and the ones the bodies
    meet (|x| < 60): equal except where both f64 values straddle an f32
    rounding midpoint (a few in 1e9), and within one f32 ulp everywhere."""
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.uniform(-60, 60, 1_500_000), rng.uniform(-2.0 ** 20, 2.0 ** 20, 500_000),
                        np.arange(-64, 65) * (np.pi / 32)]).astype(np.float32)
    s, c = batch.probe_sincos(x)
    want_s = np.sin(x.astype(np.float64)).astype(np.float32)
    want_c = np.cos(x.astype(np.float64)).astype(np.float32)
    diff = int(np.sum(s != want_s) + np.sum(c != want_c))
    assert diff <= 3, diff
    assert np.all(np.abs(s.view(np.int32).astype(np.int64) - want_s.view(np.int32)) <= 1)
    assert np.all(np.abs(c.view(np.int32).astype(np.int64) - want_c.view(np.int32)) <= 1)


def test_device_wrap_is_atan2_of_sin_and_cos():
    """readProprio's Math.atan2(Math.sin(d), Math.cos(d)), which the device
    evaluates as d wrapped into (-pi, pi], against numpy's f64 chain: 3 M
    differences of f32 angles up to 1e5 rad apart, values next to odd
    multiples of pi and arguments beyond 2^20 (where the device evaluates
    the chain itself).  Within 4 f64 ulp, and the same f32 after the
    proprioception's scalings (/ 0.42 pi for the curl, / 0.62 pi for the
    shoulder); NaN for non-finite input."""
    rng = np.random.default_rng(11)
    parts = []
    for r in (1.0, 4.0, 60.0, 1e3, 1e5):
        a = rng.uniform(-r, r, 600_000).astype(np.float32)
        b = rng.uniform(-r, r, 600_000).astype(np.float32)
        parts.append(a.astype(np.float64) - b.astype(np.float64))
    odd = (2 * np.arange(-2000, 2001) + 1) * np.pi
    parts.append((odd[:, None] + np.linspace(-1e-9, 1e-9, 11)[None, :] * (np.abs(odd[:, None]) + 1)).ravel())
    parts.append(rng.uniform(2.0 ** 20, 2.0 ** 30, 1000) * rng.choice([-1.0, 1.0], 1000))
    d = np.concatenate(parts)
    got = batch.probe_wrap(d)
    want = np.arctan2(np.sin(d), np.cos(d))
    assert np.all(np.abs(got - want) <= 4 * np.spacing(np.abs(want)))
    for scale in (0.42 * np.pi, 0.62 * np.pi):
        assert np.array_equal((got / scale).astype(np.float32), (want / scale).astype(np.float32))
    assert np.all(np.isnan(batch.probe_wrap(np.array([np.nan, np.inf, -np.inf]))))


@pytest.mark.parametrize("slice_ms", [0.0, 0.5])
def test_engine_rollouts_equal_oracle_rollout_loop_f32(slice_ms):
    """The engine's rollouts (control streams, reflex, step, postStep on the
    device; uneven horizons) against the oracle's C rollout loop with the f32
    emulation's step (xpbd_bench.c): final mantle positions bit for bit, path
    length and score within 1e-9 (f64 libm calls on both sides), in one
    launch and in time slices."""
    w = workloads.uneven(n=48, n_maps=6, seed=23, h_min=100, h_max=200)
    eng = batch.BatchEngine(w.maps, w.n)
    workloads.spawn_all(eng, w)
    eng.set_slice(slice_ms)
    eng.run(int(w.horizon.max()))
    met = eng.read_metrics()
    eng.close()
    _, _, ref = ob.bench_rollouts(w.maps, w.map_id, w.arms, w.segs, w.x, w.y, w.angle, w.seed, w.horizon, 2,
                                  metrics=True, f32=True)
    F = batch.METRIC_FIELDS
    assert np.array_equal(met[:, [F.index("x"), F.index("y")]], ref[:, :2])
    got = met[:, [F.index("pathLen"), F.index("score")]]
    assert np.all(np.abs(got - ref[:, 2:4]) <= 1e-9 * np.maximum(1.0, np.abs(ref[:, 2:4])))
