/*
 * xpbd_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of Kraken 3's XPBD creature step, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg to check and to
 * time the CUDA path.  Nothing under kraken_3_gpu_b200/ links or loads it.
 *
 * Two restatements over one world object:
 *   ref64  -- src/physics/xpbd.js (FP64, JS semantics: `%` = fmod, Math.hypot)
 *   ref32  -- tools/f32solver.mjs, collMode 'seq' (every op rounded to f32,
 *             sin/cos as (float)cos((double)x), WGSL `%` with an f64 quotient)
 * plus the builders around them: src/world/map.js (mulberry32, makeMap,
 * makeSdf, findSpawn), src/body/kraken.js (spawnKraken generalised over the
 * arm and segment count, tipPosition, attachGrip, releaseGrip,
 * toneToCompliance, adhesionToBreakForce), src/sim/core.js (createSim
 * colouring, groupConstraintsByColor, applyControl, readProprio) and
 * src/physics/xpbd.js:98-126 (assignColor, ensureColored).
 */
#ifndef KRAKEN_XPBD_ORACLE_H
#define KRAKEN_XPBD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_C_PIN 0
#define OR_C_ANGLE 1
#define OR_C_GRIP 2
#define OR_MAX_COLORS 16
#define OR_MAX_ARMS 16
#define OR_MAX_SEGS 16

/* constraint field ids for or_con_get / or_con_set (makeConstraint, xpbd.js:160-179) */
enum {
  OR_F_TYPE = 0, OR_F_A, OR_F_B, OR_F_LAX, OR_F_LAY, OR_F_LBX, OR_F_LBY,
  OR_F_COMPLIANCE, OR_F_LAMBDA, OR_F_LAMBDAX, OR_F_LAMBDAY, OR_F_BROKEN,
  OR_F_BREAKFORCE, OR_F_FORCE, OR_F_TARGET, OR_F_REST, OR_F_MINANGLE,
  OR_F_MAXANGLE, OR_F_OWNER, OR_F_COLOR, OR_F_COUNT
};

/* body array ids for or_world_array (XpbdWorld fields, xpbd.js:199-209) */
enum {
  OR_A_PX = 0, OR_A_PY, OR_A_PPX, OR_A_PPY, OR_A_VX, OR_A_VY, OR_A_ANG,
  OR_A_ANGP, OR_A_AV, OR_A_IM, OR_A_II, OR_A_FX, OR_A_FY, OR_A_TQ, OR_A_COUNT
};

typedef struct or_world or_world;
typedef struct or_sim or_sim;

/* ---- map.js ---------------------------------------------------------- */
uint32_t or_mulberry32_next(uint32_t *state, double *out);
double or_rnd(uint32_t *state);
int or_make_map(double width, double height, double wall, int cols, int rows,
                double density, uint32_t seed, double *out_rects, int max_rects);
int or_sdf(const double *rects, int n, double x, double y,
           double *d, double *nx, double *ny);
void or_find_spawn(const double *rects, int n, double width, double height,
                   double clearance, uint32_t *rng, double *x, double *y);

/* ---- XpbdWorld -------------------------------------------------------- */
or_world *or_world_new(int substeps, int iterations, double h, double linDrag,
                       double angDrag, double maxSpeed, double maxAngSpeed);
void or_world_free(or_world *w);
int or_world_n(const or_world *w);
int or_world_nc(const or_world *w);
int or_world_np(const or_world *w);
double *or_world_array(or_world *w, int which);
int or_add_body(or_world *w, double x, double y, double angle, double mass, double inertia);
void or_add_collision_point(or_world *w, int body, double lx, double ly, double r);
void or_get_collision_point(const or_world *w, int i, int *body, double *lx, double *ly, double *r);
int or_add_constraint(or_world *w, int type, int a, int b, double lax, double lay,
                      double lbx, double lby, double compliance);
double or_con_get(const or_world *w, int id, int field);
void or_con_set(or_world *w, int id, int field, double v);
int or_world_list(const or_world *w, int k);          /* solve order -> id */
void or_world_set_list(or_world *w, const int *ids, int n);
void or_world_set_rects(or_world *w, const double *rects, int n);
void or_world_color_info(const or_world *w, uint32_t *off16, uint32_t *cnt16);
void or_world_stats(const or_world *w, double *maxSpeed, double *maxAngSpeed,
                    int *nan, long *collisions, int *broken);

int or_assign_color(uint32_t *mask, int a, int b);
int or_assign_color_n(uint32_t *mask, int n, int a, int b);
void or_ensure_colored(or_world *w);
void or_group_by_color(or_world *w);

void or_step(or_world *w);              /* XpbdWorld.step, xpbd.js:487-490 */
void or_substep(or_world *w);           /* xpbd.js:257-328 */
void or_solve_collisions(or_world *w);  /* xpbd.js:447-469 */

/* ---- f32solver.mjs ---------------------------------------------------- */
void or_f32ify(or_world *w);            /* snapshot statics (f32solver.mjs:63-112) */
void or_f32_round_state(or_world *w);   /* roundState, f32solver.mjs:128-135 */
void or_step32(or_world *w);            /* patched step, f32solver.mjs:430-434 */
uint64_t or_f32_op_count(void);         /* f32 rounding ops (opcount build only) */
void or_f32_op_count_reset(void);

/* ---- kraken.js + core.js --------------------------------------------- */
typedef struct {
  int mantle, nArms, nSegs;
  int segs[OR_MAX_ARMS][OR_MAX_SEGS];
  int motors[OR_MAX_ARMS][OR_MAX_SEGS];  /* constraint ids: [0] shoulder motor */
  int grip[OR_MAX_ARMS];                  /* constraint id */
  int tip[OR_MAX_ARMS];
  double relAng[OR_MAX_ARMS];
  double spawnX, spawnY, spawnAngle;
} or_kraken;

int or_spawn_kraken(or_world *w, double x, double y, double angle, int arms,
                    int segs, double curl, or_kraken *out);
void or_tip_position(const or_world *w, const or_kraken *k, int arm, double *x, double *y);
void or_attach_grip(or_world *w, const or_kraken *k, int arm, double breakForce);
void or_release_grip(or_world *w, const or_kraken *k, int arm);
double or_tone_to_compliance(double tone);
double or_adhesion_to_break_force(double a);
double or_arm_reach(int segs);

/* createSim (core.js:37-74): world + map + creatures, coloured and grouped */
or_sim *or_sim_create(uint32_t seed, int creatures, double width, double height,
                      int substeps, int iterations, double h, int arms, int segs);
or_sim *or_sim_new(double width, double height, const double *rects, int nR, int substeps,
                   int iterations, double h);
int or_sim_add_creature(or_sim *s, double x, double y, double angle, int arms, int segs);
void or_sim_free(or_sim *s);
or_world *or_sim_world(or_sim *s);
int or_sim_rects(const or_sim *s, double *out, int max);
int or_sim_ncreatures(const or_sim *s);
void or_sim_kraken(const or_sim *s, int i, or_kraken *out);
void or_sim_set_reflex(or_sim *s, double gripSlipMax, double gripCooldown);
/* applyControl (core.js:183-220) with per-arm shoulder/curl/adhesion */
void or_apply_control(or_sim *s, int ci, double tone, const double *shoulder,
                      const double *curl, const double *adhesion);
/* the same reflex with one target per motor (arm-major, motor 0 = shoulder) */
void or_apply_control_motors(or_sim *s, int ci, double tone, const double *targets,
                             const double *adhesion);
void or_sim_reflex_state(const or_sim *s, int ci, double *cd, double *adhesion);
int or_read_proprio(or_sim *s, int ci, double *out);
void or_sim_step(or_sim *s);        /* world.step() of the whole sim */
void or_sim_step32(or_sim *s);      /* f32 emulation step */

/* fitness metrics of a creature: postStep's accumulators (core.js:297-356)
 * and score (fitness.js:115-172) */
typedef struct {
  double score, steps, pathLen, maxDisplacement, spawnReach, angularAccum, forwardProg, gripPullProg;
  double anchoredSteps, freeMove, energySpent, gripCycles, strides, attachEvents, x, y;
  double spawnDistMax;
} or_metrics;
double or_measure_reach(const double *rects, int nR, double reach, double x, double y);
void or_sim_set_spawn_reach(or_sim *s, int ci, double reach);
void or_sim_pre_step(or_sim *s);    /* preStep of every creature */
void or_sim_post_step(or_sim *s);   /* postStep of every creature */

/* the trainer's controller: senses without entities, net.js, trainStep */
typedef struct or_net_sim or_net_sim;
or_net_sim *or_net_new(or_sim *s, const double *lights, int nL);  /* lights: x y r ir ph sp */
void or_net_free(or_net_sim *n);
int or_net_param_count(int arms);
void or_net_forward(const float *w, const float *x, float *out, float *scratch, int nIn, int nOut);
int or_net_step(or_net_sim *n, const float *genomes, int n_params, const int *ind, int f32);
void or_net_io(const or_net_sim *n, int ci, float *x, float *out);
void or_net_echo(const or_net_sim *n, int ci, int *emits, int *pending);
double or_score(const or_metrics *m);

/* The timed CPU baseline (xpbd_bench.c): creatures [0, n), each in its own
 * one-creature world on map map_id[c] (rects of all maps x y w h, map_off
 * n_maps + 1), driven per env step by its mulberry32 control stream (redrawn
 * every `period` steps), applyControl, preStep, step (FP64) and postStep, to
 * its horizon or until limit_s seconds (0: none) have passed; `threads`
 * POSIX threads over contiguous ranges of about equal work.  Returns 0 and
 * the creature-steps done and the seconds from the start of the first
 * thread to the end of the last; out (n x 4, may be NULL) receives each
 * creature's final mantle x, y, path length and score (fitness.js, spawn
 * reach measured at the spawn point).  f32: step with the f32 emulation. */
int or_bench_rollouts(int n, const double *rects, const int *map_off, const int *map_id, const int *arms,
                      const int *segs, const double *x, const double *y, const double *angle,
                      const uint32_t *seed, const int *horizon, double tone, int period, int substeps,
                      int iterations, double h, double width, double height, int threads, double limit_s,
                      int f32, long long *steps_done, double *elapsed_s, double *out);
void or_sim_metrics(const or_sim *s, int ci, or_metrics *out);

#ifdef __cplusplus
}
#endif
#endif
