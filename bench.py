#!/usr/bin/env python
"""Creature-steps/s of Kraken 3's XPBD creature step on B200, persistent and
served, beside the plain per-step launch; p50/p99 rollout latency.

Workload (default): 16,384 creatures on 64 maps, bodies of 4-8 arms x 5-9
segments, horizons U{200..2000} env steps, controls from per-creature
mulberry32 streams redrawn every 6 steps (tone 0.5), S=2 substeps x I=4
iterations at h = 1/120 -- seeded synthetic data in the shapes of the
uneven-batching configuration.

value: one bench step = one full rollout of every creature to its horizon by
the persistent kernel (one launch, autotuned launch shape), state restored
from a device snapshot, L2 flushed in between; creature-steps / device time.

e2e: the same workload served through the rollout server's C ABI with host
buffers -- one request per creature (its pose, control stream and horizon),
results copied back -- with p50/p99 rollout latency.

Beside them: the plain form (the same kernel, one launch per env step), its
CUDA-graph replay, an ES request stream (Poisson 200 req/s, mirrored
populations 8-512, horizons 300-3000, fused policy MLP) through a
16,384-slot server with p50/p99 latency, the FP32-issue roofline of the
kernel and the CPU oracle (FP64 restatement of the reference's xpbd.js) on
the host cores as a reported baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "creature-steps/s at 16k mixed envs, served vs plain launch; p50/p99 rollout ms"
# DRAM bytes (read + write) of one persistent launch per creature, from a one-kernel,
# one-launch ncu capture of an 8,192-creature case (20,806,656 B read + 381,184 B written):
# the committed state, grips, controls and slot records in and out once, independent of the
# step count
NCU_DRAM_BYTES_PER_CREATURE = (20806656 + 381184) / 8192
UNIT = "creature-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--maps", type=int, default=64)
    ap.add_argument("--hmin", type=int, default=200)
    ap.add_argument("--hmax", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--shape", default="", help="lanes,warps,ctas[,unroll] launch shape (empty: autotune)")
    ap.add_argument("--chunk", type=int, default=64, help="server env steps per round (two-partition rounds)")
    ap.add_argument("--slice-ms", type=float, default=50.0,
                    help="server time slices (ms) of the one-partition scheduler; 0: two partitions in rounds")
    ap.add_argument("--engine-slice-ms", type=float, default=50.0,
                    help="persistent rollouts in preemptible time slices of this many ms, the creatures regrouped "
                         "between them (0: one launch per rollout)")
    ap.add_argument("--no-es", action="store_true", help="skip the ES request stream")
    ap.add_argument("--es-requests", type=int, default=200)
    ap.add_argument("--no-config1", action="store_true", help="skip the 1,024-creature drop-in comparison")
    ap.add_argument("--no-net", action="store_true", help="skip the reference-net controller rollout")
    ap.add_argument("--no-config4", action="store_true", help="skip the 65,536-creature memory-bound serving case")
    ap.add_argument("--net-only", action="store_true",
                    help="only the reference-net controller rollout of the workload (one JSON line)")
    ap.add_argument("--no-policy", action="store_true", help="skip the fused-policy controller rollout")
    ap.add_argument("--policy-only", action="store_true",
                    help="only the fused-policy controller rollout of the workload (one JSON line)")
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu DRAM bytes per launch of the captured kernel, if measured")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)
        self.p = None

    def start(self, wait_s: float = 3.0):
        """Starts nvidia-smi and returns once its first sample is in the file
        or wait_s has passed, so that its start-up (NVML initialisation, which
        overlapped and slowed the first timed rollout) is over before
        anything is timed."""
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        t0 = time.time()
        while time.time() - t0 < wait_s and self.p.poll() is None:
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.strip().split(",") for r in self.f.read().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU oracle (the reported baseline and the reference arm)
# ---------------------------------------------------------------------------
def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_rollouts(w, every: int, offset: int, threads: int, limit_s: float):
    """The FP64 oracle (the restated xpbd.js) on the host cores with no
    Python in the loop (oracle/xpbd_bench.c): the creatures i = offset (mod
    every) of the workload, each in its own one-creature world on its map,
    driven by its own control stream (the same mulberry32 draws the device
    makes), applyControl with the reflex, the step and postStep, to its
    horizon or until limit_s; POSIX threads over contiguous ranges of about
    equal work.  Returns (creature-steps / s, creature-steps, seconds, creatures)."""
    from oracle import binding as ob
    sel = np.arange(offset % every, w.n, every)
    steps, el = ob.bench_rollouts(w.maps, w.map_id[sel], w.arms[sel], w.segs[sel], w.x[sel], w.y[sel],
                                  w.angle[sel], w.seed[sel], w.horizon[sel], threads, limit_s=limit_s)
    return steps / el, steps, el, len(sel)


def cpu_model() -> str:
    """The host CPU's model name (Linux /proc/cpuinfo), or the platform's."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline_line(w, threads: int, seconds: float):
    """cpu_baseline of the bench line: every 32nd creature of the workload on
    all host threads (bounded by `seconds`), and the single-thread rate on
    every 512th for the per-core scaling."""
    v1, n1, e1, c1 = cpu_rollouts(w, 512, 0, 1, max(2.0, seconds / 3))
    vt, nt, et, ct = cpu_rollouts(w, 32, 0, threads, seconds)
    return {"value": vt, "unit": UNIT, "cores": threads, "kind": "port", "cpu_model": cpu_model(),
            "sample": f"{nt} creature-steps in {et:.1f} s: {ct} creatures (every 32nd) of the same workload "
                      "at their own horizons, each in its own world, controls + reflex + FP64 step + postStep "
                      "(C restatement of src/physics/xpbd.js and core.js, POSIX threads, no Python in the loop)",
            "single_thread": {"value": v1, "creature_steps": n1, "seconds": round(e1, 3), "creatures": c1},
            "scaling_vs_single_thread": vt / (threads * v1)}


def ops_per_creature_step(w, sample: int = 48, steps: int = 60) -> float:
    """f32 rounding ops per creature-step of the restated f32 algorithm
    (tools/f32solver.mjs, collMode seq) on a sample of the workload's bodies
    and maps: the algorithmic work the roofline divides by."""
    from kraken_3_gpu_b200.workloads import TONE, ControlStream
    from oracle import binding as ob

    L = ob.lib(opcount=True)
    total_ops, total_steps = 0, 0
    idx = np.linspace(0, w.n - 1, sample).astype(int)
    for i in idx:
        sim = ob.Sim(rects=w.maps[w.map_id[i]], opcount=True)
        sim.add_creature(w.x[i], w.y[i], w.angle[i], int(w.arms[i]), int(w.segs[i]))
        sim.world.f32ify()
        sim.world.round_state()
        cs = ControlStream(int(w.arms[i]), int(w.segs[i]), seed=int(w.seed[i]))
        L.or_f32_op_count_reset()
        for s in range(steps):
            tg, ad = cs.at(s)
            sim.apply_control_motors(0, TONE, tg, ad)
            sim.step32()
        total_ops += L.or_f32_op_count()
        total_steps += steps
    # weight by each creature's horizon share is unnecessary: the sample is
    # spread evenly over the workload
    return total_ops / total_steps


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_env():
    from kraken_3_gpu_b200 import replicas
    return replicas.dist_env()


def bench_config(args, w, world: int) -> dict:
    """The workload description both arms print (the same dict, so the two
    lines describe one configuration)."""
    return {"workload": f"uneven-{w.n}: {w.n:,} creatures, {len(w.maps)} maps, 4-8 arms x 5-9 segments, "
                        f"horizons {args.hmin}-{args.hmax}",
            "creatures": w.n, "maps": len(w.maps), "creature_steps_per_rollout": w.creature_steps(),
            "seed": args.seed, "substeps": 2, "iterations": 4,
            "controls": "per-creature mulberry32 streams, redraw every 6 steps, reflex on",
            "parallelism": f"contiguous creature ranges of one workload x{world}" if world > 1 else "1 GPU",
            "l2": "GPU arm: flushed between timed rollouts (256 MB write), state restored from a device "
                  "snapshot inside the timed region"}


def reference_arm(args):
    """The reference's algorithm on the host cores: the FP64 oracle (the
    reference is browser JavaScript; no JS runtime here) driven as the GPU
    arm drives its creatures, on the same workload realisation.  One bench
    step = one bounded sample of it: the creatures i = step (mod 32) at their
    own horizons, on every host thread, at most 20 s."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from kraken_3_gpu_b200 import replicas, workloads
    w = workloads.uneven(n=args.n, n_maps=args.maps, seed=args.seed,
                         h_min=args.hmin, h_max=args.hmax)
    threads = host_threads()
    for k in range(args.warmup):
        cpu_rollouts(w, 32, 31 - k, threads, 2.0)
    total, el, ms = 0, 0.0, []
    for k in range(args.steps):
        _, n, e, _ = cpu_rollouts(w, 32, k, threads, 20.0)
        total += n
        el += e
        ms.append(e * 1000)
    value = total / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": float(np.mean(ms)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args, w, world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"per step the creatures i = step (mod 32) of the workload ({w.n // 32:,}) at "
                                   "their own horizons, at most 20 s; FP64 restatement of src/physics/xpbd.js with "
                                   "core.js's applyControl and postStep in C on POSIX threads (the reference is "
                                   "browser JavaScript, no JS runtime on the box)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def served_uneven(serve, w, chunk, sessions, slice_ms=0.0):
    """The mixed workload through the rollout server's C ABI with host
    buffers: one request per creature (its own pose, control stream and
    horizon), all submitted at once; results read back to the host.  The
    server picks each round's launch shape from its partition's live count."""
    srv = serve.Server(w.maps, 8 << 30, max_slots=w.n, chunk_steps=chunk if slice_ms <= 0 else 1 << 20,
                       policy=False, slice_ms=slice_ms)
    xs, ys, an = (np.ascontiguousarray(v, dtype=np.float64) for v in (w.x, w.y, w.angle))
    seeds = np.ascontiguousarray(w.seed, dtype=np.uint32)
    out = []
    for _ in range(sessions):
        s0 = srv.stats()
        t0 = time.perf_counter()
        ids = srv.submit_many(w.horizon, w.arms, w.segs, w.map_id, xs, ys, an, control_seeds=seeds)
        srv.drain()
        res, times = srv.results_many(ids, release=True)
        wall = time.perf_counter() - t0
        s1 = srv.stats()
        out.append({"wall_s": wall, "lat": times[:, 2] - times[:, 0],
                    "h2d": s1["h2d_bytes"] - s0["h2d_bytes"], "d2h": s1["d2h_bytes"] - s0["d2h_bytes"],
                    "device_ms": s1["device_ms"] - s0["device_ms"],
                    "host_gap_ms": s1["host_gap_ms"] - s0["host_gap_ms"], "slices": s1["rounds"] - s0["rounds"]})
    srv.close()
    return out


def served_es_stream(serve, w, chunk, n_req, rate, seed=0, net=False, slice_ms=0.0):
    """ES evaluation requests (mirrored populations 8-512, horizons
    300-3000, body shapes and maps of the mixed workload, fused policy with
    theta ~ N(0, 0.1^2), sigma 0.02) arriving as a Poisson stream.  net: the
    requests' theta is a genome of the reference net (net.js), which then
    drives every individual with its senses."""
    rng = np.random.default_rng(seed)
    reqs, t = [], 0.0
    for k in range(n_req):
        t += rng.exponential(1.0 / rate)
        i = int(rng.integers(0, w.n))
        arms, segs = int(w.arms[i]), int(w.segs[i])
        reqs.append(dict(population=2 * int(rng.integers(4, 257)), horizon=int(rng.integers(300, 3001)),
                         arms=arms, segs=segs, map_id=int(w.map_id[i]), x=float(w.x[i]), y=float(w.y[i]),
                         angle=float(w.angle[i]),
                         theta=rng.normal(0, 0.1, serve.net_param_count(arms) if net else
                                          serve.policy_params(arms, segs)).astype(np.float32),
                         sigma=0.02, seed=k + 1, arrival=t))
    units = sum(r["population"] * r["horizon"] for r in reqs)
    kw = dict(max_slots=16384, chunk_steps=chunk if slice_ms <= 0 else 1 << 20, slice_ms=slice_ms)
    srv = (serve.Server(w.maps, 8 << 30, net=True, lights=w.lights, **kw) if net
           else serve.Server(w.maps, 8 << 30, policy=True, **kw))
    t0 = srv.now() + 0.02
    ids = []
    for r in reqs:
        r = dict(r)
        r["arrival"] += t0
        ids.append(srv.submit(**r))
    srv.drain()
    res = [srv.result(i, r["population"]) for i, r in zip(ids, reqs)]
    st = srv.stats()
    srv.close()
    lat = np.array([x["completed"] - x["arrival"] for x in res])
    queue = np.array([x["admitted"] - x["arrival"] for x in res])
    service = np.array([x["completed"] - x["admitted"] for x in res])
    span = max(x["completed"] for x in res) - min(x["arrival"] for x in res)
    arrivals = reqs[-1]["arrival"] - reqs[0]["arrival"]

    def pct(a, q):
        return float(np.percentile(a, q) * 1e3)

    return {"value": units / span, "unit": UNIT, "requests": n_req, "rate_req_s": rate,
            "offered_rate": units / max(arrivals, 1e-9), "delivered_rate": units / span,
            "creature_steps": units, "makespan_s": span, "arrivals_span_s": arrivals,
            "p50_rollout_ms": pct(lat, 50), "p99_rollout_ms": pct(lat, 99),
            "queue_p50_ms": pct(queue, 50), "queue_p99_ms": pct(queue, 99),
            "service_p50_ms": pct(service, 50), "service_p99_ms": pct(service, 99),
            "slots": st["capacity"], "chunk_steps": chunk if slice_ms <= 0 else None,
            "slice_ms": slice_ms if slice_ms > 0 else None, "rounds_or_slices": st["rounds"],
            "host_gap_ms": st["host_gap_ms"],
            "device_kernel_ms_summed": st["device_ms"]}


def served_es_streams(serve, w, chunk, n_req, rate, net=False, slice_ms=0.0):
    """The configured stream (Poisson `rate` req/s: it offers more work than
    one GPU delivers, so its latencies grow with the stream's length), and the
    same request mix at a sustainable load: the Poisson rate scaled so that the
    offered creature-steps/s are 0.8 x the rate the first stream delivered
    (the server's capacity under this mix)."""
    over = served_es_stream(serve, w, chunk, n_req, rate, net=net, slice_ms=slice_ms)
    sus_rate = rate * 0.8 * over["delivered_rate"] / over["offered_rate"]
    sus = served_es_stream(serve, w, chunk, n_req, sus_rate, net=net, slice_ms=slice_ms)
    over["sustainable_load"] = sus
    return over


def config1_forms(torch, stream, steps=1000):
    """The plain batched drop-in configuration: 1,024 default creatures on
    map seed 1, spawn jitter U(+-20 px) around the map's spawn point, heading
    U[0, 2 pi), 1,000 env steps, random controls per creature (its own
    control stream, redrawn every 6 steps).  Two forms on the same creatures
    and controls: the reference's plain loop through the drop-in (HybridLoop:
    per env step the reflex on the host, the 80 B constraint blocks up, one
    kr_step, bodies and constraints down), timed whole and by the kernel time
    of its steps; and the persistent batched engine (reflex and controls on the
    device, one launch).  The persistent engine runs the same arithmetic, so
    the two forms' final states are compared bit for bit as well."""
    from kraken_3_gpu_b200 import batch, hybrid, workloads
    w = workloads.uniform(n=1024, steps=steps)
    loop = hybrid.HybridLoop(w, stream.cuda_stream)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(steps):
        loop.step(evs[k])
    loop_s = time.perf_counter() - t0
    kernel_ms = sum(a.elapsed_time(b) for a, b in evs)
    mant = [c.mantle for c in loop.sim["creatures"]]
    dropin_xy = loop.body[mant][:, :2].copy()
    cons_bytes, body_bytes = loop.g.consData.nbytes, loop.g.bodyData.nbytes
    loop.close()
    eng = batch.BatchEngine(w.maps, w.n)
    eng.set_stream(stream.cuda_stream)
    workloads.spawn_all(eng, w)
    eng.snapshot()
    g, wp, c, _ = eng.autotune(64)
    eng.restore()
    eng.run(64)
    eng.restore()
    eng.run(steps)
    eng.sync()
    pers_ms = eng.last_ms()
    st = eng.read_state()
    shape = eng.get_launch()
    eng.close()
    pers_xy = np.stack([st["px"][:, 0], st["py"][:, 0]], axis=1)
    same = float(np.mean(np.all(pers_xy.astype(np.float32) == dropin_xy, axis=1)))
    n = w.n
    return {"creatures": n, "map_seed": 1, "steps": steps,
            "dropin_per_step_loop": {"value": n * steps / loop_s, "unit": UNIT,
                                     "form": "reference plain loop: host reflex + packControls, uploadControls, "
                                             "kr_step, download, per env step",
                                     "h2d_bytes_per_step": int(cons_bytes),
                                     "d2h_bytes_per_step": int(cons_bytes + body_bytes)},
            "dropin_per_step_kernel": {"value": n * steps / (kernel_ms / 1000.0), "unit": UNIT,
                                       "kernel_ms": kernel_ms,
                                       "form": "the kr_step launches of that loop alone (CUDA events)"},
            "persistent": {"value": n * steps / (pers_ms / 1000.0), "unit": UNIT, "kernel_ms": pers_ms,
                           "launch_shape": [shape["lanes_per_creature"], shape["warps_per_cta"],
                                            shape["ctas_per_sm"], shape["substep_unroll"]]},
            "persistent_over_dropin_kernel": (n * steps / (pers_ms / 1000.0)) / (n * steps / (kernel_ms / 1000.0)),
            "final_mantles_bit_identical": same}


def config4_memory_bound(serve, slice_ms):
    """The memory-bound configuration: 65,536 creatures of the mixed bodies
    (64 maps, horizons U{200..4096}), each with a 128-step observation ring,
    one request per creature submitted at once to a server whose slot count
    comes from its HBM budget: 8 GB (every creature fits: 33.5 KB per slot
    with the ring) and 1.5 GB (about 47,800 slots, so requests queue for
    slots freed by completed ones).  Wall clock per run, results copied back."""
    from kraken_3_gpu_b200 import workloads
    w = workloads.uneven(n=65536, n_maps=64, seed=4, h_min=200, h_max=4096)
    xs, ys, an = (np.ascontiguousarray(v, dtype=np.float64) for v in (w.x, w.y, w.angle))
    out = {"creatures": w.n, "creature_steps": w.creature_steps(), "obs_ring": 128}
    for name, budget in (("budget_8GB", 8 << 30), ("budget_1.5GB", int(1.5 * (1 << 30)))):
        srv = serve.Server(w.maps, budget, policy=False, obs_ring=128, chunk_steps=1 << 20 if slice_ms > 0 else 128,
                           slice_ms=slice_ms)
        t0 = time.perf_counter()
        ids = srv.submit_many(w.horizon, w.arms, w.segs, w.map_id, xs, ys, an, control_seeds=w.seed)
        srv.drain()
        res, times = srv.results_many(ids, release=True)
        wall = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        lat = times[:, 2] - times[:, 0]
        out[name] = {"value": w.creature_steps() / wall, "unit": UNIT, "wall_s": wall, "slots": st["capacity"],
                     # requests not admitted with the first ones: they waited for freed slots
                     "queued_requests": int(np.sum(times[:, 1] > times[:, 1].min() + 1e-3)),
                     "p50_rollout_ms": float(np.percentile(lat, 50) * 1e3),
                     "p99_rollout_ms": float(np.percentile(lat, 99) * 1e3), "slices_or_rounds": st["rounds"],
                     "host_gap_ms": st["host_gap_ms"], "device_bytes": st["device_bytes"]}
    return out


def policy_controller(stream, w, seed=8, slice_ms=0.0, shape=None):
    """The same workload driven by the fused policy MLP (KR_CTRL_POLICY, the
    ES requests' controller: proprioception -> 64 tanh -> motor targets and
    adhesion), one individual per creature with its own weights theta ~
    N(0, 0.1^2) in its body shape's layout -- every creature reads its own
    weights each env step, as an ES population's individuals do; the whole
    horizons with the autotuned launch shape (or `shape`: lanes, warps, CTAs
    per SM[, unroll]), in time slices of slice_ms (0: one launch), device time
    by CUDA events."""
    from kraken_3_gpu_b200 import batch, workloads
    rng = np.random.default_rng(seed)
    width = max(batch.policy_params(int(a), int(g)) for a, g in zip(w.arms, w.segs))
    weights = np.zeros((w.n, width), np.float32)
    for i in range(w.n):
        k = batch.policy_params(int(w.arms[i]), int(w.segs[i]))
        weights[i, :k] = rng.normal(0, 0.1, k)
    eng = batch.BatchEngine(w.maps, w.n, control="policy")
    eng.set_stream(stream.cuda_stream)
    workloads.spawn_all(eng, w)
    eng.set_policy(weights, np.arange(w.n, dtype=np.int32))
    eng.snapshot()
    if shape:
        eng.set_launch(shape[1], shape[2], lanes_per_creature=shape[0])
        if len(shape) > 3:
            eng.set_unroll(shape[3])
    else:
        eng.autotune(64)  # the launch shape, as the persistent bench picks it; slots left as they were
    eng.set_slice(slice_ms)
    eng.run(64)
    eng.restore()
    eng.run(int(w.horizon.max()))
    eng.sync()
    ms = eng.last_ms()
    shape = eng.get_launch()
    slices = eng.last_slices()
    eng.close()
    return {"value": w.creature_steps() / (ms / 1000.0), "unit": UNIT, "kernel_ms": ms,
            "controller": "fused policy MLP 6A+6 -> 64 tanh -> A*S+A per creature, its own weights (theta ~ N(0, 0.1^2))",
            "launch_shape": [shape["lanes_per_creature"], shape["warps_per_cta"], shape["ctas_per_sm"],
                             shape["substep_unroll"]],
            "time_slices": slices, "slice_ms": slice_ms if slice_ms > 0 else None}


def net_controller(stream, w, seed=7, slice_ms=0.0):
    """The same workload driven by the reference trainer's own controller
    (KR_CTRL_NET: net.js's recurrent net on proprioception + echo, light and
    contact senses), one randomGenome-initialised genome per creature (net.js:
    41-55: N(0, 1/fan_in) weights, zero biases); the whole horizons with the
    autotuned launch shape, in time slices of slice_ms (0: one launch), device
    time by CUDA events."""
    from kraken_3_gpu_b200 import batch, workloads
    rng = np.random.default_rng(seed)
    width = batch.net_param_count(int(w.arms.max()))
    genomes = np.zeros((w.n, width), np.float32)
    H = batch.NET_HIDDEN
    for i in range(w.n):
        A = int(w.arms[i])
        ni, no = batch.net_inputs(A), batch.net_outputs(A)
        k = 0
        for n, s in ((ni * H, 1 / np.sqrt(ni)), (H, 0.0), (H * H, 1 / np.sqrt(H)), (H, 0.0),
                     (H * no, 1 / np.sqrt(H)), (no, 0.0)):
            genomes[i, k:k + n] = rng.normal(0, 1, n) * s
            k += n
    eng = batch.BatchEngine(w.maps, w.n, control="net", lights=w.lights)
    eng.set_stream(stream.cuda_stream)
    workloads.spawn_all(eng, w)
    eng.set_net(genomes, np.arange(w.n, dtype=np.int32))
    eng.snapshot()
    eng.autotune(64)  # the launch shape, as the persistent bench picks it; slots left as they were
    eng.set_slice(slice_ms)
    eng.run(64)
    eng.restore()
    eng.run(int(w.horizon.max()))
    eng.sync()
    ms = eng.last_ms()
    shape = eng.get_launch()
    slices = eng.last_slices()
    eng.close()
    return {"value": w.creature_steps() / (ms / 1000.0), "unit": UNIT, "kernel_ms": ms,
            "controller": "net.js 10A+45 -> 24 -> 24 -> 3A+2 per creature, senses and recurrent outputs on the device",
            "launch_shape": [shape["lanes_per_creature"], shape["warps_per_cta"], shape["ctas_per_sm"],
                             shape["substep_unroll"]],
            "time_slices": slices, "slice_ms": slice_ms if slice_ms > 0 else None}


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch

    from kraken_3_gpu_b200 import batch, replicas, serve, workloads

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    # one explicit stream for the engine, the events and the copies
    torch.cuda.set_stream(torch.cuda.Stream())
    replicas.init("nccl", world, local)

    def barrier():
        replicas.barrier(world)

    def all_max(x: float) -> float:
        return replicas.max_over_ranks(x, world)

    # one workload of world x n creatures, contiguous ranges of n per rank
    # (rank 0's range is the one-GPU workload)
    w_all = workloads.uneven(n=args.n * world, n_maps=args.maps, seed=args.seed, h_min=args.hmin, h_max=args.hmax)
    w, (lo, hi) = replicas.shard(w_all, rank, world)
    del w_all
    if args.net_only or args.policy_only:
        if args.net_only:
            line = net_controller(torch.cuda.current_stream(), w, slice_ms=args.engine_slice_ms)
            line["metric"] = "creature-steps/s under the reference net controller"
        else:
            shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else None
            line = policy_controller(torch.cuda.current_stream(), w, slice_ms=args.engine_slice_ms, shape=shape)
            line["metric"] = "creature-steps/s under the fused policy controller"
        line.update({"n_gpus": 1, "config": {"workload": f"uneven: {w.n} creatures, {len(w.maps)} maps, horizons "
                                                         f"{args.hmin}-{args.hmax}"}})
        if rank == 0:
            print(json.dumps(line))
        replicas.finish(world)
        return
    units = w.creature_steps()
    max_h = int(w.horizon.max())
    stream = torch.cuda.current_stream()
    eng = batch.BatchEngine(w.maps, w.n)
    eng.set_stream(stream.cuda_stream)
    workloads.spawn_all(eng, w)
    eng.snapshot()
    # L2 flush between timed rollouts (a write larger than the 126 MB L2);
    # written once here so that its kernel is loaded before anything is timed
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    flush.zero_()

    # autotune the launch shape (lanes per creature, warps per CTA, CTAs per
    # SM) on a 64-step slice of the workload; every shape gives the same bits
    tune = {}
    if args.shape:
        best = tuple(int(v) for v in args.shape.split(","))
        eng.set_launch(best[1], best[2], lanes_per_creature=best[0])
        if len(best) > 3:
            eng.set_unroll(best[3])
        best = best[:3]
    else:
        g, wp, c, ms = eng.autotune(64)  # the library's autotuner: slots left as they were
        best = (g, wp, c)
        tune = {best: ms}
    unroll = eng.get_launch()["substep_unroll"]
    eng.set_slice(args.engine_slice_ms)
    shape_choice = None
    if args.engine_slice_ms > 0 and not args.shape:
        # the autotuner times 64 steps of the whole population; a sliced
        # rollout also runs the tail, where the automatic shape of each slice
        # (more lanes per creature as creatures finish) may be faster: two
        # whole rollouts with each, the faster kept (untimed, as warm-up)
        def rollout_ms():
            eng.restore()
            eng.run(max_h)
            eng.sync()
            return eng.last_ms()

        t_tuned = min(rollout_ms(), rollout_ms())
        eng.set_launch(0, 0, lanes_per_creature=0)
        t_auto = min(rollout_ms(), rollout_ms())
        shape_choice = {"autotuned_ms": round(t_tuned, 3), "automatic_ms": round(t_auto, 3)}
        if t_tuned <= t_auto:
            eng.set_launch(best[1], best[2], lanes_per_creature=best[0])
        else:
            best = ("automatic per slice",) * 3
        shape_choice["kept"] = "autotuned" if t_tuned <= t_auto else "automatic"

    # warm-up: full rollouts, each as a timed one runs
    for _ in range(args.warmup):
        flush.zero_()
        eng.restore()
        eng.run(max_h)
    barrier()

    sampler = ClockSampler(local)
    sampler.start()
    # one more rollout while the sampler starts: the GPU stays busy (and its
    # clocks up) until the timed region begins
    eng.restore()
    eng.run(max_h)
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    gpu_launches = 0
    for k in range(args.steps):
        flush.zero_()
        eng.restore()
        eng.run(max_h)
        ev[k + 1].record(stream)
        slices, kernels, creature_launches = eng.last_run_launches()
        gpu_launches += kernels
    ev[-1].synchronize()
    barrier()
    e0, e1 = ev[0], ev[-1]
    rollout_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    elapsed_ms = e0.elapsed_time(e1)
    # the last rollout's launches (events on its stream; under time slices
    # from its first slice to its last, the host time between them included)
    kms = eng.last_ms()
    t_max = all_max(elapsed_ms)
    value = replicas.job_rate(units * args.steps, world, t_max / 1000.0)
    ms_per_step = t_max / args.steps

    extra = {}
    # the edge of the partition: every rank's per-creature scores gathered in
    # workload order (one all-gather, outside the timed region)
    scores = eng.read_metrics()[:, 0]
    counts = [replicas.contiguous_range(args.n * world, r, world)[1] - replicas.contiguous_range(args.n * world, r, world)[0]
              for r in range(world)]
    gathered = replicas.gather_fitness(scores, counts, world, device="cuda")
    extra["partition"] = {"creatures": [lo, hi], "ranks": world, "gathered_scores": int(gathered.size),
                          "gathered_score_sum": float(np.sum(gathered))}
    # plain form: the same kernel, one launch per env step
    if not args.no_plain:
        eng.restore()
        torch.cuda.synchronize()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        eng.run_launches(1, max_h)
        p1.record(stream)
        p1.synchronize()
        plain_ms = all_max(p0.elapsed_time(p1))
        extra["plain_per_step_launch"] = {"value": world * units / (plain_ms / 1000.0), "unit": UNIT,
                                          "ms_per_rollout": plain_ms, "launches": max_h}
        eng.restore()
        eng.run_graph(1, max_h, 1)
        g_ms = all_max(eng.last_ms())
        extra["graph_step_loop"] = {"value": world * units / (g_ms / 1000.0), "unit": UNIT,
                                    "ms_per_rollout_replay": g_ms, "launches_in_graph": max_h}

    # end to end: the workload served through the rollout server's C ABI with
    # host buffers (requests in, results out), p50/p99 rollout latency
    chunk, sl = args.chunk, args.slice_ms

    def served_line(slice_ms):
        sess = served_uneven(serve, w, chunk, 1 + max(1, min(args.steps, 2)), slice_ms=slice_ms)[1:]
        wall = all_max(sum(x["wall_s"] for x in sess))
        lat = np.concatenate([x["lat"] for x in sess])
        return {"value": world * units * len(sess) / wall, "unit": UNIT,
                "h2d_bytes_per_step": int(np.mean([x["h2d"] for x in sess])),
                "d2h_bytes_per_step": int(np.mean([x["d2h"] for x in sess])),
                "p50_rollout_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_rollout_ms": float(np.percentile(lat, 99) * 1e3),
                "slices_or_rounds_per_session": float(np.mean([x["slices"] for x in sess])),
                "host_gap_ms_per_session": float(np.mean([x["host_gap_ms"] for x in sess]))}

    e2e = served_line(sl)
    clocks = sampler.stop()
    e2e["form"] = ("served: rollout server C ABI, one request per creature, host buffers in and out; " +
                   (f"one partition in preemptible slices of {sl:g} ms, completions polled every 1 ms"
                    if sl > 0 else
                    f"two partitions in rounds of {chunk} env steps"))
    if sl > 0:
        extra["served_two_partitions"] = dict(served_line(0.0), chunk_steps=chunk,
                                              form="the same, two partitions in rounds of chunk_steps")

    # the engine's own host-buffer API: spawn from host arrays (poses,
    # shapes, horizons, seeds), one kr_batch_run (in time slices, as the timed
    # rollouts), the metrics record read back -- per rollout, wall-clock
    # through the C ABI
    if rank == 0:
        reps = []
        for _ in range(3):
            t0 = time.perf_counter()
            workloads.spawn_all(eng, w)
            eng.run(max_h)
            m = eng.read_metrics()
            reps.append(time.perf_counter() - t0)
        extra["engine_api_e2e"] = {
            "value": units / min(reps[1:]), "unit": UNIT,
            "form": "batched engine C ABI: kr_batch_spawn from host arrays, kr_batch_run (time slices as the timed "
                    "rollouts), kr_batch_read_metrics",
            # the library's staging of each spawned creature: its pose block (6 x 76 f32), slot record
            # (184 B) and slot index; the metrics record back
            "h2d_bytes_per_step": int(w.n * (6 * 76 * 4 + 184 + 4)), "d2h_bytes_per_step": int(m.nbytes),
            "wall_s": [round(x, 4) for x in reps]}

    if not args.no_es and rank == 0:
        extra["served_es_stream"] = served_es_streams(serve, w, chunk, args.es_requests, 200.0, slice_ms=sl)
    if not args.no_config1 and rank == 0:
        extra["plain_dropin_1024"] = config1_forms(torch, stream)
    if not args.no_config4 and rank == 0:
        extra["memory_bound_65k"] = config4_memory_bound(serve, sl)
    if not args.no_policy and rank == 0:
        extra["policy_controller"] = policy_controller(stream, w, slice_ms=args.engine_slice_ms)
    if not args.no_net and rank == 0:
        extra["net_controller"] = net_controller(stream, w, slice_ms=args.engine_slice_ms)
        if not args.no_es:
            extra["served_es_stream_net"] = served_es_streams(serve, w, chunk, args.es_requests, 200.0, net=True,
                                                              slice_ms=sl)

    # roofline: f32 rounding ops per creature-step of the restated f32
    # algorithm (op-counting oracle build) x creature-steps per launch /
    # launch duration, against the measured dependent-free FMA issue rate
    roof = None
    cpu = None
    if rank == 0:
        fma_rate = batch.probe_fp32_rate()
        if not args.no_cpu_baseline and world == 1:
            ops = ops_per_creature_step(w)
            achieved = ops * units / (kms / 1000.0)
            n_sm = torch.cuda.get_device_properties(local).multi_processor_count
            nominal = {f"{mhz:g}_mhz": n_sm * 128 * mhz * 1e6 / 1e12
                       for mhz in sorted({clocks["sm_max_mhz"] or 1965.0, clocks["sm_mhz"] or 1965.0})}
            roof = {"bound": "fp32", "achieved": achieved / 1e12, "peak": fma_rate / 1e12,
                    "unit": "TFLOP/s", "frac": achieved / fma_rate,
                    "peak_nominal": nominal,
                    "frac_nominal": {k: achieved / (v * 1e12) for k, v in nominal.items()},
                    "peak_nominal_note": f"{n_sm} SMs x 128 FP32 lanes x SM clock, at the maximum and at the median "
                                         "clock sampled under load",
                    "traffic": (args.traffic if args.traffic is not None
                                else NCU_DRAM_BYTES_PER_CREATURE * creature_launches),
                    "traffic_note": "per rollout, as achieved: ncu dram__bytes_read.sum + dram__bytes_write.sum per "
                                    "creature of a one-launch capture (8,192 creatures: 2,587 B each: state, grips, "
                                    "controls and slot records in and out once per launch) x the creatures the "
                                    f"rollout's {slices} launch(es) ran ({creature_launches}); algorithmic ~2.5 KB "
                                    "per creature per launch",
                    "ops_per_creature_step": ops, "kernel_ms": kms,
                    "kernel_ms_note": (f"the rollout's {slices} time-slice launches of batch_kernel, first to last, "
                                       "the host time between them included" if slices > 1 else
                                       "the rollout's one launch of batch_kernel"),
                    "peak_note": "measured dependent-free f32 FMA issue rate (lane-ops/s) of this GPU; "
                                 "MEASURED_PEAKS.json has no f32 figure"}
            cpu = cpu_baseline_line(w, host_threads(), args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "rollout_ms": [round(x, 3) for x in rollout_ms],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": bench_config(args, w, world),
            "form": ("persistent kernel, state resident in HBM; " +
                     (f"each rollout in preemptible time slices of {args.engine_slice_ms:g} ms, the live creatures "
                      "regrouped between slices" if slices > 1 else "one launch per rollout")),
            "launch": {"lanes_per_creature": best[0], "warps_per_cta": best[1], "ctas_per_sm": best[2],
                       "substep_unroll": unroll, "time_slices_per_rollout": slices, "shape_choice": shape_choice,
                       "slice_ms": args.engine_slice_ms if slices > 1 else None,
                       "autotune_ms": {",".join(map(str, k)): round(v, 3) for k, v in tune.items()}},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks, "e2e": e2e,
            "gpu_launches": gpu_launches, **extra,
        }
        print(json.dumps(line), flush=True)
    eng.close()
    replicas.finish(world)


if __name__ == "__main__":
    main()
