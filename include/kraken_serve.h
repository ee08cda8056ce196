/*
 * kraken_serve.h -- device-resident rollout server on B200 (sm_100a).
 *
 * Serves ES evaluation requests: a request is a mirrored population of
 * creatures of one body shape on one map, spawned at a common pose, run for
 * `horizon` env steps, each individual controlled by the fused policy MLP of
 * kraken_batch.h with its own parameters theta + sigma * eps_k (even
 * individual 2k) or theta - sigma * eps_k (odd 2k + 1), eps_k ~ N(0, 1) drawn
 * on the device from the request's seed -- the mirrored sampling of the
 * reference's ES (src/brain/es.js:67-81) -- or, without theta, by control
 * streams from the seed.  The reference evaluates a population in lockstep
 * through its hybrid loop (src/sim/gputrain.js:72-150); here requests arrive
 * at any time and share the GPU:
 *
 *  - continuous batching (slice_ms = 0): the slots are split into two partitions that run
 *    alternately on two streams, chunk_steps env steps per round; a request
 *    that arrives while others run is admitted at the next round of a
 *    partition as soon as slots are free, and its creatures run in the same
 *    launches as everyone else's (one partition's launch fills the tail of
 *    the other's);
 *  - or (slice_ms > 0) one partition in preemptible slices: a slice runs
 *    every live creature to its horizon and ends early when an arrived
 *    request fits the free slots or its time is up; the next slice admits
 *    and regroups the creatures by their remaining steps.  Requests whose
 *    creatures have all ended complete while the slice runs;
 *  - admission against an HBM budget: every slot's device memory (state,
 *    grips, controls, observation ring, policy weights) is accounted for at
 *    creation; the budget fixes the slot count, requests wait in FIFO order
 *    until enough slots are free;
 *  - per-request completion: a request's results are gathered on the device
 *    and copied back when its last round ends (slices: within about a
 *    millisecond of its last creature's end); its slots return to the pool.
 *
 * Every creature's trajectory depends only on its own request (body, map,
 * pose, parameters, seed), so a request's results are bit-identical whether
 * it runs alone or in any mix, in any slots, in either partition.
 *
 * Plain pointers and sizes; every call returns KR_OK (0) or a KR_ERR_* code
 * of kraken_b200.h; the handle is not thread-safe (one host thread drives
 * it).  Times are seconds on the server's clock (kr_server_now).
 */
#ifndef KRAKEN_SERVE_H
#define KRAKEN_SERVE_H
#include <stdint.h>

#include "kraken_b200.h"
#include "kraken_batch.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kr_server kr_server;

typedef struct kr_server_desc {
  kr_solver_params solver;      /* shared by all creatures */
  int32_t n_maps;               /* >= 1 */
  const float *rects;           /* every map's rects, x y w h (f32) */
  const int32_t *map_rect_off;  /* n_maps + 1 offsets into rects (in rects) */
  uint64_t hbm_budget_bytes;    /* device memory the server may hold */
  int32_t max_slots;            /* cap on concurrent creatures (0: what the budget allows) */
  int32_t obs_ring;             /* steps of each creature's observation ring (0: none) */
  int32_t chunk_steps;          /* env steps of a partition per round (>= 1) */
  int32_t policy;               /* 1: keep fused-policy weights per slot (requests with theta) */
  int32_t lanes_per_creature;   /* launch shape, kr_batch_set_launch (0: defaults) */
  int32_t warps_per_cta;
  int32_t ctas_per_sm;
  double grip_slip_max;         /* px/s, core.js:30 */
  double grip_cooldown;         /* s, core.js:31 */
  /* 1: requests with theta run the reference trainer's own controller
   * (KR_CTRL_NET of kraken_batch.h) -- theta is a net.js genome for the
   * request's arm count, perturbed per individual exactly as the fused
   * policy's theta is; needs policy == 0.  lights / map_light_off / map_size
   * as in kr_batch_desc; NULL lights: none. */
  int32_t net;
  const double *lights;
  const int32_t *map_light_off;
  const double *map_size;
  /* > 0: sliced scheduling instead of the two partitions' rounds.  All
   * slots form one partition and every creature runs to its horizon in one
   * persistent launch (a slice, at most chunk_steps env steps).  While it
   * runs, the server copies back the kernel's per-request counts of
   * creatures at their horizons once a millisecond and completes the
   * requests whose creatures have all ended (their records copied back
   * beside the running kernel).  It preempts the slice -- through a device
   * word the kernel reads at each env step -- when an arrived request fits
   * the free slots plus those of the completed requests (not before the
   * slice has run 10 times the host's time between slices) or slice_ms
   * milliseconds (at least 10 such host gaps) have passed, then frees the
   * completed requests' slots, admits, and launches the next slice, its
   * creatures regrouped by their remaining steps (the longest spread over
   * every SM: a shorter tail than one launch).
   * 0: two partitions alternating chunk_steps rounds (above). */
  double slice_ms;
} kr_server_desc;

typedef struct kr_request {
  int32_t population;           /* individuals, >= 1 (mirrored pairs: even) */
  int32_t horizon;              /* env steps, >= 1 */
  int32_t arms, segs;           /* body shape (1..8 x 1..9) */
  int32_t map_id;
  double x, y, angle;           /* common spawn pose (spawnKraken, src/body/kraken.js:64-101) */
  const double *xs, *ys, *angles;     /* or one pose per individual (all three, or NULL) */
  const uint32_t *control_seeds;      /* no theta: stream seed per individual (NULL: from seed) */
  float tone;                   /* muscle tone 0..1 */
  const float *theta;           /* NULL: control streams; else n_params floats (kraken_batch.h policy
                                   layout, or with net: a net.js genome, kr_batch_set_net) */
  int32_t n_params;
  float sigma;
  uint64_t seed;                /* eps (policy) or control streams (no theta) */
  double arrival;               /* server time the request arrives (< 0: now) */
  /* Index of this request's first individual in a population split over
   * several servers (one per GPU): individual i here is individual
   * first_individual + i of the whole population -- its mirrored pair
   * (first_individual + i) / 2, its sign, and without theta its control
   * stream -- so the split population's results equal the whole one's.
   * Even, >= 0; 0 for a whole population. */
  int32_t first_individual;
} kr_request;

/* results per individual: the metrics record of kraken_batch.h
 * (KR_METRIC_WORDS f64: the reference's score first, then postStep's
 * accumulators, the final mantle position last) */
#define KR_RESULT_WORDS KR_METRIC_WORDS

typedef struct kr_server_stats {
  int32_t capacity;             /* slots */
  int32_t partition_capacity;   /* slots one partition may hold */
  int32_t live;                 /* creatures on the device */
  int32_t queued;               /* requests waiting for admission */
  int64_t submitted, admitted, completed, rounds;
  double creature_steps;        /* env steps run by every admitted creature so far */
  double device_ms;             /* summed kernel time of the rounds */
  uint64_t bytes_per_slot;      /* device bytes of one slot */
  uint64_t device_bytes;        /* device bytes the server holds */
  uint64_t h2d_bytes;           /* host-to-device bytes copied so far (spawns, weights, schedules) */
  uint64_t d2h_bytes;           /* device-to-host bytes copied so far (results) */
  double host_gap_ms;           /* sliced scheduling: summed host time between a slice's end and the next launch */
} kr_server_stats;

/* The slot count and per-slot bytes a descriptor yields (no device needed). */
int kr_server_plan(const kr_server_desc *d, int32_t *capacity, uint64_t *bytes_per_slot);

int kr_server_create(const kr_server_desc *d, kr_server **out);
double kr_server_now(const kr_server *s);

/* Queue a request (theta is copied); *id identifies it.  Rejects a
 * population larger than a partition, an unknown map or body shape, and a
 * theta shorter than the body's policy needs. */
int kr_server_submit(kr_server *s, const kr_request *r, int64_t *id);

/* kr_server_submit for n requests in one call; stops at the first rejected
 * request (its status is returned), *n_submitted = requests queued. */
int kr_server_submit_batch(kr_server *s, const kr_request *reqs, int32_t n, int64_t *ids,
                           int32_t *n_submitted);

/* One scheduling step.  Two partitions (slice_ms = 0): the next partition's
 * round -- wait for its previous round, complete the requests that ended
 * there, admit arrived requests into free slots, launch chunk_steps env
 * steps of its creatures.  Slices (slice_ms > 0): while a slice runs,
 * complete the requests it has finished (at most one poll a millisecond)
 * and, unless an arrived request fits or the slice's time is up, return;
 * otherwise end the slice (preempting it if needed), free, admit and
 * launch the next one.
 * *busy = 1 while any request is queued or running. */
int kr_server_pump(kr_server *s, int32_t *busy);

/* Pump until every submitted request has completed (sleeps while the next
 * request has not arrived yet, and 0.1 ms between looks at a running slice). */
int kr_server_drain(kr_server *s);

/* Ids of requests completed since the last poll (up to cap). */
int kr_server_poll(kr_server *s, int64_t *ids, int32_t cap, int32_t *n);

/* Results of a completed request: population x KR_RESULT_WORDS f64, and
 * times[3] = arrival, admission and completion (server clock).  Either
 * pointer may be NULL. */
int kr_server_result(kr_server *s, int64_t id, double *results, double *times);

/* kr_server_result for n completed requests: results concatenated in id
 * order (sum of populations x KR_RESULT_WORDS f64), times n x 3; with
 * release != 0 the requests are forgotten afterwards. */
int kr_server_result_batch(kr_server *s, const int64_t *ids, int32_t n, double *results, double *times,
                           int32_t release);

/* Forget a completed request. */
int kr_server_release(kr_server *s, int64_t id);

int kr_server_get_stats(kr_server *s, kr_server_stats *out);

/* The first n normal numbers eps(seed, pair, 0..n) the device draws for
 * mirrored pair `pair` of a request (synchronous; for checking). */
int kr_policy_eps(uint64_t seed, int32_t pair, int32_t n, float *out);

/* Stops a running slice at its creatures' next env step (a round of two
 * partitions runs to its end), waits for the device and frees everything;
 * requests not yet completed are dropped.  NULL is a no-op. */
void kr_server_destroy(kr_server *s);
const char *kr_server_last_error(const kr_server *s);

#ifdef __cplusplus
}
#endif
#endif
