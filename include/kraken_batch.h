/*
 * kraken_batch.h -- batched creature engine on B200 (sm_100a).
 *
 * Many independent creatures of uneven body shape, on many maps, each with
 * its own horizon, advanced by one persistent kernel per call: one warp per
 * creature, creatures of one body shape grouped per CTA, a device work queue
 * over the groups.  The suction-cup reflex (applyControl, src/sim/core.js:
 * 183-220) and the proprioception vector (readProprio, core.js:129-175) run
 * on the device in f64, exactly as the reference's hybrid trainer runs them
 * on the CPU over the f32 GPU state (src/sim/gputrain.js:72-128), so every
 * creature behaves bit for bit like a one-creature gpuworld.js world driven
 * by that loop.
 *
 * Per env step and creature: proprioception of the current state -> obs ring
 * (optional) -> controls (device stream, host buffer or fused policy) ->
 * reflex -> substeps x iterations of the XPBD step -> grip break.
 *
 * Plain pointers and sizes; every call returns KR_OK (0) or a KR_ERR_* code
 * of kraken_b200.h; the handle is not thread-safe (one host thread, one
 * stream).
 */
#ifndef KRAKEN_BATCH_H
#define KRAKEN_BATCH_H
#include <stdint.h>

#include "kraken_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

#define KR_BATCH_MAX_ARMS 8
#define KR_BATCH_MAX_SEGS 9
#define KR_OBS_STRIDE 56   /* 6 * arms + 6 proprio values (f32), ..., word 55 = grip flags */

/* control sources */
#define KR_CTRL_STREAM 0   /* per-creature mulberry32 stream, redrawn every period steps */
#define KR_CTRL_BUFFER 1   /* host-provided buffer, one record per creature (kr_batch_set_controls) */
#define KR_CTRL_POLICY 2   /* fused per-creature MLP on the proprioception vector */
#define KR_CTRL_NET 3      /* the reference trainer's own recurrent net on proprioception + senses */

/* KR_CTRL_NET sizes: net.js's HIDDEN, echo.js's ECHO_RAYS, lights per map
 * (at most), and the strides of kr_batch_read_net */
#define KR_NET_HIDDEN 24
#define KR_NET_RAYS 12
#define KR_NET_MAX_LIGHTS 8
#define KR_NET_IN_STRIDE 128
#define KR_NET_OUT_STRIDE 32

typedef struct kr_batch kr_batch;

typedef struct kr_batch_desc {
  kr_solver_params solver;     /* shared by all creatures */
  int32_t n_maps;              /* >= 1 */
  const float *rects;          /* every map's rects, x y w h (f32) */
  const int32_t *map_rect_off; /* n_maps + 1 offsets into rects (in rects) */
  int32_t capacity;            /* creature slots */
  int32_t obs_ring;            /* steps kept in each creature's observation ring (0: none) */
  double grip_slip_max;        /* px/s, core.js:30 */
  double grip_cooldown;        /* s, core.js:31 */
  int32_t control_mode;        /* KR_CTRL_* */
  int32_t control_period;      /* KR_CTRL_STREAM: steps between redraws (>= 1) */
  /* KR_CTRL_NET only (NULL otherwise): every map's moving lights as makeMap
   * draws them (src/world/map.js:60-69), x y r ir ph sp per light (f64),
   * map_light_off (n_maps + 1 offsets, in lights, at most KR_NET_MAX_LIGHTS
   * per map) and map_size (n_maps x width, height: the lights' clamp).
   * NULL lights: no lights (the light sense reads the ambient level). */
  const double *lights;
  const int32_t *map_light_off;
  const double *map_size;
} kr_batch_desc;

int kr_batch_create(const kr_batch_desc *desc, kr_batch **out);

/* Spawn (or respawn) creatures into slots [first, first + n): body shape
 * arms x segs, the spawnKraken pose at (x, y, angle) (src/body/kraken.js:
 * 64-101), zero velocity, every grip released, motor targets 0, muscle tone
 * `tone` (compliance 1 / (2000 + tone * 398000), kraken.js:186-191), step
 * counter 0 and the given horizon; control_seed seeds the slot's control
 * stream (mulberry32, src/world/map.js:11-20).  Asynchronous. */
int kr_batch_spawn(kr_batch *b, int32_t first, int32_t n, const int32_t *arms,
                   const int32_t *segs, const int32_t *map_id, const double *x, const double *y,
                   const double *angle, const int32_t *horizon, const uint32_t *control_seed,
                   const float *tone);

/* KR_CTRL_BUFFER: the control record of every slot, capacity x record floats,
 * record = arms * segs motor targets (arm-major, shoulder first) then arms
 * adhesion values, laid out at stride KR_BATCH_MAX_ARMS * (KR_BATCH_MAX_SEGS + 1).
 * Copied host->device on the handle's stream; used by every following step
 * until replaced. */
int kr_batch_set_controls(kr_batch *b, const float *controls);

/* KR_CTRL_POLICY: the fused controller of every slot.  weights holds
 * n_individuals parameter vectors of n_params floats each; slot s uses
 * vector slot_individual[s] (capacity entries).  Layout per vector, row-major
 * with the bias last: W1 (KR_POLICY_HIDDEN x (n_in + 1)) then W2
 * (n_out x (KR_POLICY_HIDDEN + 1)), n_in = 6 * arms + 6 (the proprioception
 * vector), n_out = arms * segs motor targets (tanh) + arms adhesion values
 * ((tanh + 1) / 2).  Copied host->device on the handle's stream. */
#define KR_POLICY_HIDDEN 64
int kr_batch_set_policy(kr_batch *b, const float *weights, int32_t n_individuals, int32_t n_params,
                        const int32_t *slot_individual);

/* KR_CTRL_NET: the reference trainer's own controller (src/sim/train.js:
 * 233-249, src/sim/gputrain.js:72-90) per slot and env step, on the device:
 * the input vector -- readProprio (6A + 6 values), readSenses (core.js:
 * 233-242: echo 2 x 12, chemoreception 6, light 3, hearing 4, tip contact A;
 * without prey or other entities the chemoreception and hearing read 0) and
 * the previous step's A_out = 3A + 2 outputs, n_in = 10A + 45 values, each
 * rounded to f32 as the trainer's Float32Array holds it -- through net.js's
 * forwardInto (src/brain/net.js:71-98: two tanh layers of KR_NET_HIDDEN and
 * a tanh output layer, f64 sums of f32 products, tanh clamped to +-1 beyond
 * +-20, activations rounded to f32), decode (net.js:124-133: tone, per arm
 * shoulder, curl and adhesion, echo emission above 0.3) and applyControl
 * with that tone.  After the XPBD step and postStep the senses advance as
 * tickSenses does (core.js:245-267): the map's lights move (tickMapLights,
 * map.js:75-83), the echo's cooldown runs and arrived echoes are written, an
 * emission marches 12 rays against the map (echo.js:67-127), the light and
 * contact senses are sampled.  A slot starts as a creature of a fresh sim:
 * time 0, lights at the positions of the map description, sense buffers
 * and recurrent outputs 0.  For A = 6 the network is net.js's 105 -> 24 ->
 * 24 -> 20 with its 3,644 weights; other arm counts use the same layout with
 * n_in = 10A + 45 and A_out outputs.
 *
 * genomes holds n_individuals weight vectors at a stride of n_params floats,
 * each in net.js's layout (weightCount: n_in x 24, 24, 24 x 24, 24, 24 x
 * A_out, A_out) for the arm count of the spawned slots that use it (its
 * first weightCount floats are read; n_params must be at least that for
 * every such slot, so one call serves bodies of several arm counts); slot s
 * uses vector slot_individual[s] (capacity entries). */
int kr_batch_set_net(kr_batch *b, const float *genomes, int32_t n_individuals, int32_t n_params,
                     const int32_t *slot_individual);

/* KR_CTRL_NET: the input vector and outputs of each slot's last env step
 * (synchronous): inputs n x KR_NET_IN_STRIDE f32 (n_in used), outputs n x
 * KR_NET_OUT_STRIDE f32 (A_out used).  Either pointer may be NULL. */
int kr_batch_read_net(kr_batch *b, int32_t first, int32_t n, float *inputs, float *outputs);

/* Advance every live slot by min(max_steps, horizon - step) env steps with
 * one persistent launch.  Asynchronous; returns once enqueued -- except
 * under time slices (kr_batch_set_slice) when max_steps covers every live
 * slot's remaining steps: then the run is a sequence of launches and the
 * call returns when every creature has reached its horizon. */
int kr_batch_run(kr_batch *b, int32_t max_steps);

/* Time slices.  slice_ms > 0: a kr_batch_run that takes every live slot to
 * its horizon runs as preemptible slices -- a persistent launch, stopped
 * through a device word after slice_ms (creatures stop at an env-step
 * boundary, state written back), the step counters read back, the live
 * creatures regrouped by their remaining steps and launched again.  The
 * regrouping spreads the longest creatures over every SM as the short ones
 * finish, so the tail of uneven horizons runs with shorter steps; the
 * results are bit-identical to one launch.  A slice that advanced no
 * creature doubles the next one's time.  0 (default): one launch.
 * kr_batch_last_ms then covers the whole run, host time between slices
 * included; kr_batch_last_slices gives the slices it took, the kernels it
 * launched (slices and step-counter readbacks; 1 and 1 for one launch) and
 * the creatures its slices launched, summed over the slices (each slice
 * loads and writes back the state of the creatures it runs).  Any pointer
 * may be NULL. */
int kr_batch_set_slice(kr_batch *b, float slice_ms);
int kr_batch_last_slices(kr_batch *b, int32_t *slices, int32_t *kernels, int64_t *creature_launches);

/* `launches` back-to-back launches of steps_per_launch env steps each over
 * the same creature groups, no host work between them (with
 * steps_per_launch = 1: the plain one-launch-per-env-step form). */
int kr_batch_run_launches(kr_batch *b, int32_t steps_per_launch, int32_t launches);

/* Capture `launches` consecutive kr_batch_run(max_steps) calls into one CUDA
 * graph and replay it `replays` times. */
int kr_batch_run_graph(kr_batch *b, int32_t max_steps, int32_t launches, int32_t replays);

/* Number of slots whose step counter is below their horizon (synchronous). */
int kr_batch_live(kr_batch *b, int32_t *live);

/* Copy the state of slots [first, first + n) to the host (synchronous):
 * bodies: n x (1 + 8 * 9) x 6 f32 (px py vx vy ang av per body, template
 * body order), grips: n x 8 x 4 f32 (lbx lby breakForce broken), steps: n
 * i32.  Any pointer may be NULL. */
int kr_batch_read_state(kr_batch *b, int32_t first, int32_t n, float *bodies, float *grips,
                        int32_t *steps);

/* Copy the observation rings of slots [first, first + n) to the host
 * (synchronous): n x obs_ring x KR_OBS_STRIDE f32, entry t % obs_ring holds
 * the proprioception read at the start of env step t. */
int kr_batch_read_obs(kr_batch *b, int32_t first, int32_t n, float *obs);

/* The controls each slot used in its last env step (synchronous): n x
 * KR_BATCH_MAX_ARMS * (KR_BATCH_MAX_SEGS + 1) f32 in the kr_batch_set_controls
 * record layout (motor controls before clamping, adhesion values). */
int kr_batch_read_controls(kr_batch *b, int32_t first, int32_t n, float *controls);

/* Per-slot accumulators (synchronous): n x 4 f64 -- path length of the
 * mantle, x and y of the mantle, attach events (arms newly anchored after a
 * step). */
int kr_batch_read_fitness(kr_batch *b, int32_t first, int32_t n, double *out);

/* The reference's fitness metrics of every slot (synchronous): n x
 * KR_METRIC_WORDS f64, accumulated on the device after every env step as
 * postStep does (src/sim/core.js:297-356, f64 on the f32 state), with the
 * score of src/sim/fitness.js:115-172 (no prey; maxAngSpeed 18, dt 1/60).
 * The spawn reach is measureReach (fitness.js:74-88) of the spawn point on
 * the map's rects as given (f32 values), rays up to 3.5 reaches of the body.
 * Words: score, steps, path length, max displacement, spawn reach, angular
 * accumulation, forward progress, grip-pull progress, anchored steps, free
 * move, energy spent, grip cycles, strides, attach events, mantle x, y. */
#define KR_METRIC_WORDS 16
int kr_batch_read_metrics(kr_batch *b, int32_t first, int32_t n, double *out);

/* Keep a device copy of every slot's state (bodies, grips, reflex
 * cooldowns, current controls, step counters) and put it back later -- the
 * snapshot/restore of a rollout; both asynchronous device-to-device copies
 * (the snapshot synchronizes once when it first allocates). */
int kr_batch_snapshot(kr_batch *b);
int kr_batch_restore(kr_batch *b);

/* Dependent-free f32 FMA throughput of the device (FMA instructions per
 * second over every SM), the issue-rate ceiling of the f32 path. */
int kr_probe_fp32_rate(double *fma_per_s);

/* The solver's sin / cos of f32 angles (Math.fround of the f64 sin / cos, as
 * f32solver.mjs evaluates them) for n host values: s[i], c[i] of x[i].
 * Synchronous; for checking the device's trig against a reference. */
int kr_probe_sincos(const float *x, int32_t n, float *s, float *c);

/* readProprio's atan2(sin d, cos d) of f64 angle differences as the device
 * evaluates it (src/body/kraken.js:173 armCurl, src/sim/core.js:138 the
 * shoulder angle): out[i] for d[i], d wrapped into (-pi, pi].
 * Synchronous; for checking the device's wrap against a reference. */
int kr_probe_wrap(const double *d, int32_t n, double *out);

/* Launch shape: lanes per creature (32, 16 or 8: a warp carries 32 / lanes
 * creatures), warps per CTA (1..16, at most 64 creatures per CTA) and CTAs
 * per SM (0 = 16 / warps).  A CTA gets an equal share of the SM's shared
 * memory; a group of one body template holds as many creatures as fit in it.
 * Until this is called the engine picks the shape per launch: 32 lanes x 4
 * warps below 16 live creatures per SM, 16 lanes x 8 warps below 96 (8
 * lanes when most creatures run the fused policy or the net, or an
 * observation ring is kept), else 8 lanes x 8 warps -- x 16 warps in one CTA
 * per SM when most creatures run the net or a ring is kept;
 * lanes_per_creature = 0 returns to that (the other arguments are
 * ignored).  Results do not depend on the launch
 * shape. */
int kr_batch_set_launch(kr_batch *b, int32_t lanes_per_creature, int32_t warps_per_cta,
                        int32_t ctas_per_sm);

/* Substep unroll: the kernel's substep loop runs as a loop (1) or with its
 * body twice per trip (2); the same operations in the same order, so the
 * results do not depend on it -- only the instruction stream does.  Default
 * 1; kr_batch_autotune picks it with the launch shape. */
int kr_batch_set_unroll(kr_batch *b, int32_t substep_unroll);
int kr_batch_get_unroll(kr_batch *b, int32_t *substep_unroll);

/* The current launch shape and the dynamic shared memory of a CTA (bytes;
 * 0 before the first spawn).  Any pointer may be NULL. */
int kr_batch_get_launch(kr_batch *b, int32_t *lanes_per_creature, int32_t *warps_per_cta,
                        int32_t *ctas_per_sm, int32_t *smem_bytes);

/* Autotuner: runs `steps` env steps of the live slots with each candidate
 * launch shape (8, 16 and 32 lanes per creature with 4-16 warps per CTA,
 * each with the substep loop rolled or unrolled by 2), puts every slot's
 * state back after each trial (slots end as they were; the
 * kr_batch_snapshot copy is not touched) and keeps the fastest shape
 * (kr_batch_set_launch, kr_batch_set_unroll).  The chosen shape and its time
 * are returned (the unroll through kr_batch_get_unroll); any pointer may be
 * NULL.  Synchronous. */
int kr_batch_autotune(kr_batch *b, int32_t steps, int32_t *lanes_per_creature, int32_t *warps_per_cta,
                      int32_t *ctas_per_sm, float *best_ms);

/* Device time of the last kr_batch_run launch in ms (synchronous). */
int kr_batch_last_ms(kr_batch *b, float *ms);

int kr_batch_sync(kr_batch *b);
int kr_batch_set_stream(kr_batch *b, void *stream);
void kr_batch_destroy(kr_batch *b);
const char *kr_batch_last_error(const kr_batch *b);

#ifdef __cplusplus
}
#endif
#endif
