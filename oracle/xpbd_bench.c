/*
 * xpbd_bench.c -- TEST INFRASTRUCTURE ONLY (the timed CPU baseline, never
 * the product).
 *
 * The loop the batched engine runs per stream-controlled creature, on the
 * host's cores with the FP64 oracle (the restated src/physics/xpbd.js), so
 * that bench.py can time it without Python in the loop:
 *   per env step t of a creature:
 *     if t % period == 0: draw the controls from the creature's mulberry32
 *       stream (src/world/map.js:11-20), per arm its motors then its
 *       adhesion, targets as r * 2 - 1 and adhesion as r, each held as f32
 *       (the controls of a Float32Array, as the engine's control record);
 *     applyControl (core.js:183-220: targets clamped, the suction-cup reflex),
 *     preStep, world.step() (xpbd.js:487-490; or, for checks, the f32
 *     emulation's step of tools/f32solver.mjs), postStep (core.js:297-356).
 * Every creature lives in its own one-creature world on its map, as the
 * reference's creatures never interact.  All worlds are built before the
 * clock starts; creatures are then split into contiguous ranges of about
 * equal work (horizon x constraint count), one POSIX thread per range, and
 * each thread runs its creatures one after the other to their horizons, or
 * until the time limit.
 */
#define _POSIX_C_SOURCE 200809L
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "xpbd_oracle.h"

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

typedef struct {
  int begin, end;                 /* creature range [begin, end) */
  or_sim **sims;                  /* one world per creature of the range */
  const int *arms, *segs, *horizon;
  const uint32_t *seed;
  double tone, deadline;
  int period;
  double *out;                    /* per creature: mantle x, y, path length, score, or NULL */
  int f32;                        /* 1: the f32 emulation's step (f32solver.mjs) instead of FP64 */
  long long steps;
  double t_end;
} bench_job;

static void *bench_thread(void *arg) {
  bench_job *J = (bench_job *)arg;
  long long done = 0;
  double tg[OR_MAX_ARMS * OR_MAX_SEGS], ad[OR_MAX_ARMS];
  int stop = 0;
  for (int c = J->begin; c < J->end && !stop; c++) {
    or_sim *s = J->sims[c - J->begin];
    const int A = J->arms[c], S = J->segs[c];
    uint32_t rng = J->seed[c];
    for (int t = 0; t < J->horizon[c] && !stop; t++) {
      if (t % J->period == 0) {
        for (int a = 0; a < A; a++) {
          for (int j = 0; j < S; j++) tg[a * S + j] = (double)(float)(or_rnd(&rng) * 2 - 1);
          ad[a] = (double)(float)or_rnd(&rng);
        }
      }
      or_apply_control_motors(s, 0, J->tone, tg, ad);
      or_sim_pre_step(s);
      if (J->f32) or_sim_step32(s);
      else or_sim_step(s);
      or_sim_post_step(s);
      done++;
      if (J->deadline > 0 && (done & 15) == 0 && now_s() > J->deadline) stop = 1;
    }
    if (J->out) {
      or_metrics m;
      or_sim_metrics(s, 0, &m);
      J->out[4 * c] = m.x;
      J->out[4 * c + 1] = m.y;
      J->out[4 * c + 2] = m.pathLen;
      J->out[4 * c + 3] = m.score;
    }
  }
  J->t_end = now_s();
  J->steps = done;
  return NULL;
}

int or_bench_rollouts(int n, const double *rects, const int *map_off, const int *map_id, const int *arms,
                      const int *segs, const double *x, const double *y, const double *angle,
                      const uint32_t *seed, const int *horizon, double tone, int period, int substeps,
                      int iterations, double h, double width, double height, int threads, double limit_s,
                      int f32, long long *steps_done, double *elapsed_s, double *out) {
  if (n < 1 || threads < 1 || period < 1 || !steps_done || !elapsed_s) return -1;
  for (int c = 0; c < n; c++)
    if (arms[c] < 1 || arms[c] > OR_MAX_ARMS || segs[c] < 1 || segs[c] > OR_MAX_SEGS || horizon[c] < 0) return -1;
  if (threads > n) threads = n;
  bench_job *J = (bench_job *)calloc((size_t)threads, sizeof(bench_job));
  pthread_t *th = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
  char *started = (char *)calloc((size_t)threads, 1);
  or_sim **sims = (or_sim **)calloc((size_t)n, sizeof(or_sim *));
  int rc = (J && th && started && sims) ? 0 : -1;
  /* every creature's world, built before the clock starts */
  for (int c = 0; c < n && rc == 0; c++) {
    const int m = map_id[c];
    sims[c] = or_sim_new(width, height, rects + 4 * (size_t)map_off[m], map_off[m + 1] - map_off[m],
                         substeps, iterations, h);
    if (!sims[c] || or_sim_add_creature(sims[c], x[c], y[c], angle[c], arms[c], segs[c]) < 0) {
      rc = -2;
      continue;
    }
    /* measureReach at the spawn point, as createSim records it for score() */
    or_sim_set_spawn_reach(sims[c], 0, or_measure_reach(rects + 4 * (size_t)map_off[m], map_off[m + 1] - map_off[m],
                                                        or_arm_reach(segs[c]), x[c], y[c]));
    if (f32) {
      or_f32ify(or_sim_world(sims[c]));
      or_f32_round_state(or_sim_world(sims[c]));
    }
  }
  double t0 = 0, t_end = 0;
  long long steps = 0;
  if (rc == 0) {
    /* contiguous ranges of about equal work: horizon x constraint count (a
       pin and an angle per segment and a grip per arm, as spawnKraken builds
       the body) */
    double total = 0, acc = 0;
    for (int c = 0; c < n; c++) total += (double)horizon[c] * (double)(arms[c] * (2 * segs[c] + 1));
    int c = 0;
    t0 = now_s();
    for (int k = 0; k < threads; k++) {
      J[k].begin = c;
      const double goal = total * (double)(k + 1) / threads;
      while (c < n && (k == threads - 1 || acc < goal)) {
        acc += (double)horizon[c] * (double)(arms[c] * (2 * segs[c] + 1));
        c++;
      }
      J[k].end = c;
      J[k].sims = sims + J[k].begin;
      J[k].arms = arms; J[k].segs = segs; J[k].horizon = horizon; J[k].seed = seed;
      J[k].tone = tone; J[k].period = period; J[k].out = out; J[k].f32 = f32;
      J[k].deadline = limit_s > 0 ? t0 + limit_s : 0;
    }
    for (int k = 0; k < threads; k++) {
      if (pthread_create(&th[k], NULL, bench_thread, &J[k]) == 0) started[k] = 1;
      else bench_thread(&J[k]);  /* no thread: run the range here */
    }
    for (int k = 0; k < threads; k++) {
      if (started[k]) pthread_join(th[k], NULL);
      steps += J[k].steps;
      if (J[k].t_end > t_end) t_end = J[k].t_end;
    }
  }
  for (int c = 0; sims && c < n; c++)
    if (sims[c]) or_sim_free(sims[c]);
  *steps_done = steps;
  *elapsed_s = t_end - t0;
  free(J);
  free(th);
  free(started);
  free(sims);
  return rc;
}
