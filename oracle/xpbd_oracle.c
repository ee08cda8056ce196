/*
 * xpbd_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * CPU restatement of the reference's XPBD step and of the builders around it.
 * Every function names the reference file:line it follows.  Two arithmetic
 * paths share one world object:
 *
 *   ref64 (or_step)   src/physics/xpbd.js -- FP64 with JavaScript semantics:
 *                     `a % b` is C fmod (exact), Math.hypot is hypot,
 *                     Number.isFinite is isfinite.
 *   ref32 (or_step32) tools/f32solver.mjs, collMode 'seq' -- every arithmetic
 *                     result rounded to f32 (Math.fround), sin/cos/exp taken
 *                     in f64 and rounded, the WGSL `%` emulated with an f64
 *                     quotient (f32solver.mjs:36-51).
 *
 * Build with -ffp-contract=off (no FMA contraction) and without -ffast-math;
 * x86-64 SSE arithmetic then rounds each float op once, like Math.fround.
 * Built with -DOR_COUNT_OPS it also counts the f32 rounding ops of ref32
 * (one per f() call of f32solver.mjs), which defines the algorithmic work
 * of one creature-step for the roofline.
 */
#include "xpbd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ======================================================================
 * constants
 * ==================================================================== */
#define JS_PI 3.141592653589793
static const double SLACK_POS = 2e-3;   /* xpbd.js:77 */
static const double SLACK_ANG = 2e-4;   /* xpbd.js:78 */

/* BODY, kraken.js:22-47 */
#define B_SEGLEN 13.5
#define B_SHOULDER_R 24.0
#define B_MANTLE_R 18.0
#define B_MANTLE_MASS 20.0
#define B_MANTLE_IF 2.5
#define B_SEG_MASS_PROX 3.2
#define B_SEG_MASS_DIST 1.8
#define B_SEG_THICK_PROX 11.9
#define B_SEG_THICK_DIST 5.9
#define B_SPAWN_CURL 0.28
#define B_STIFF_MIN 2000.0
#define B_STIFF_MAX 400000.0
#define B_GRIP_MIN 40.0
#define B_GRIP_MAX 900.0
static double joint_limit(void) { return JS_PI * 0.42; }
static double shoulder_limit(void) { return JS_PI * 0.62; }

/* ======================================================================
 * world object
 * ==================================================================== */
typedef struct {
  int type, a, b;
  double lax, lay, lbx, lby, compliance;
  double lambda, lambdaX, lambdaY;
  int broken;
  double breakForce, force, target, rest, minAngle, maxAngle;
  int owner, color;
} orc_t;

typedef struct {
  int active;
  float h, invH, invH2, linDamp, angDamp, maxSpeed, maxAngSpeed;
  int n, nC, nR, nP;
  float *imF, *iiF;
  float *laxF, *layF, *restF, *minF, *maxF;
  int *typeArr, *aArr, *bArr, *conId;
  float *rx, *ry, *rxw, *ryh;
  int *cpBody;
  float *cpLx, *cpLy, *cpR;
  int *bpOff, *bpCnt, *bpIdx;
  float *compF, *tgtF, *lbxF, *lbyF, *brkF;
} f32snap_t;

struct or_world {
  int substeps, iterations;
  double h, linDrag, angDrag, maxSpeed, maxAngSpeed;
  int n, cap;
  double *arr[OR_A_COUNT];
  int nP, capP;
  int *cpBody;
  double *cpLx, *cpLy, *cpR;
  int nC, capC;
  orc_t *cons;   /* creation order: stable ids (JS object identity) */
  int *list;     /* solve order: list[k] = id (XpbdWorld.constraints) */
  int nR;
  double *rects; /* x, y, w, h per rect; nR == 0 and no sdf => no collisions */
  int hasSdf;
  double st_maxSpeed, st_maxAngSpeed;
  int st_nan, st_broken;
  long st_collisions;
  int colored;
  uint32_t colorOff[OR_MAX_COLORS], colorCnt[OR_MAX_COLORS], colorMax;
  f32snap_t f;
};

#define PX(w) ((w)->arr[OR_A_PX])
#define PY(w) ((w)->arr[OR_A_PY])
#define PPX(w) ((w)->arr[OR_A_PPX])
#define PPY(w) ((w)->arr[OR_A_PPY])
#define VX(w) ((w)->arr[OR_A_VX])
#define VY(w) ((w)->arr[OR_A_VY])
#define ANG(w) ((w)->arr[OR_A_ANG])
#define ANGP(w) ((w)->arr[OR_A_ANGP])
#define AV(w) ((w)->arr[OR_A_AV])
#define IM(w) ((w)->arr[OR_A_IM])
#define II(w) ((w)->arr[OR_A_II])
#define FX(w) ((w)->arr[OR_A_FX])
#define FY(w) ((w)->arr[OR_A_FY])
#define TQ(w) ((w)->arr[OR_A_TQ])

/* XpbdWorld constructor, xpbd.js:189-214 */
or_world *or_world_new(int substeps, int iterations, double h, double linDrag,
                       double angDrag, double maxSpeed, double maxAngSpeed) {
  or_world *w = (or_world *)calloc(1, sizeof(or_world));
  w->substeps = substeps;
  w->iterations = iterations;
  w->h = h;
  w->linDrag = linDrag;
  w->angDrag = angDrag;
  w->maxSpeed = maxSpeed;
  w->maxAngSpeed = maxAngSpeed;
  return w;
}

static void f32_free(f32snap_t *f) {
  void *ptrs[] = {f->imF, f->iiF, f->laxF, f->layF, f->restF, f->minF, f->maxF,
                  f->typeArr, f->aArr, f->bArr, f->conId, f->rx, f->ry, f->rxw,
                  f->ryh, f->cpBody, f->cpLx, f->cpLy, f->cpR, f->bpOff, f->bpCnt,
                  f->bpIdx, f->compF, f->tgtF, f->lbxF, f->lbyF, f->brkF};
  for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
  memset(f, 0, sizeof(*f));
}

void or_world_free(or_world *w) {
  if (!w) return;
  for (int i = 0; i < OR_A_COUNT; i++) free(w->arr[i]);
  free(w->cpBody); free(w->cpLx); free(w->cpLy); free(w->cpR);
  free(w->cons); free(w->list); free(w->rects);
  f32_free(&w->f);
  free(w);
}

int or_world_n(const or_world *w) { return w->n; }
int or_world_nc(const or_world *w) { return w->nC; }
int or_world_np(const or_world *w) { return w->nP; }
double *or_world_array(or_world *w, int which) {
  return (which >= 0 && which < OR_A_COUNT) ? w->arr[which] : NULL;
}

/* _grow, xpbd.js:230-240 */
static void grow(or_world *w) {
  int cap = w->cap * 2 > 64 ? w->cap * 2 : 64;
  for (int i = 0; i < OR_A_COUNT; i++) {
    double *d = (double *)calloc((size_t)cap, sizeof(double));
    if (w->arr[i]) memcpy(d, w->arr[i], sizeof(double) * (size_t)w->cap);
    free(w->arr[i]);
    w->arr[i] = d;
  }
  w->cap = cap;
}

/* addBody, xpbd.js:217-228 */
int or_add_body(or_world *w, double x, double y, double angle, double mass, double inertia) {
  int i = w->n++;
  if (i >= w->cap) grow(w);
  PX(w)[i] = x; PY(w)[i] = y;
  PPX(w)[i] = x; PPY(w)[i] = y;
  VX(w)[i] = 0; VY(w)[i] = 0;
  ANG(w)[i] = angle; ANGP(w)[i] = angle; AV(w)[i] = 0;
  IM(w)[i] = mass > 0 ? 1 / mass : 0;
  II(w)[i] = inertia > 0 ? 1 / inertia : 0;
  FX(w)[i] = 0; FY(w)[i] = 0; TQ(w)[i] = 0;
  return i;
}

/* addCollisionPoint, xpbd.js:243-245 */
void or_add_collision_point(or_world *w, int body, double lx, double ly, double r) {
  if (w->nP >= w->capP) {
    int cap = w->capP * 2 > 64 ? w->capP * 2 : 64;
    w->cpBody = (int *)realloc(w->cpBody, sizeof(int) * (size_t)cap);
    w->cpLx = (double *)realloc(w->cpLx, sizeof(double) * (size_t)cap);
    w->cpLy = (double *)realloc(w->cpLy, sizeof(double) * (size_t)cap);
    w->cpR = (double *)realloc(w->cpR, sizeof(double) * (size_t)cap);
    w->capP = cap;
  }
  w->cpBody[w->nP] = body;
  w->cpLx[w->nP] = lx;
  w->cpLy[w->nP] = ly;
  w->cpR[w->nP] = r;
  w->nP++;
}

void or_get_collision_point(const or_world *w, int i, int *body, double *lx, double *ly, double *r) {
  *body = w->cpBody[i]; *lx = w->cpLx[i]; *ly = w->cpLy[i]; *r = w->cpR[i];
}

/* makeConstraint (xpbd.js:160-179) + addConstraint (xpbd.js:247) */
int or_add_constraint(or_world *w, int type, int a, int b, double lax, double lay,
                      double lbx, double lby, double compliance) {
  if (w->nC >= w->capC) {
    int cap = w->capC * 2 > 64 ? w->capC * 2 : 64;
    w->cons = (orc_t *)realloc(w->cons, sizeof(orc_t) * (size_t)cap);
    w->list = (int *)realloc(w->list, sizeof(int) * (size_t)cap);
    w->capC = cap;
  }
  orc_t *c = &w->cons[w->nC];
  memset(c, 0, sizeof(*c));
  c->type = type; c->a = a; c->b = b;
  c->lax = lax; c->lay = lay; c->lbx = lbx; c->lby = lby;
  c->compliance = compliance;
  c->lambda = 0; c->lambdaX = 0; c->lambdaY = 0;
  c->broken = 0;
  c->breakForce = INFINITY;
  c->force = 0;
  c->target = 0;
  c->rest = 0;
  c->minAngle = -INFINITY;
  c->maxAngle = INFINITY;
  c->owner = -1;
  c->color = -1;
  w->list[w->nC] = w->nC;
  return w->nC++;
}

double or_con_get(const or_world *w, int id, int field) {
  const orc_t *c = &w->cons[id];
  switch (field) {
    case OR_F_TYPE: return c->type;
    case OR_F_A: return c->a;
    case OR_F_B: return c->b;
    case OR_F_LAX: return c->lax;
    case OR_F_LAY: return c->lay;
    case OR_F_LBX: return c->lbx;
    case OR_F_LBY: return c->lby;
    case OR_F_COMPLIANCE: return c->compliance;
    case OR_F_LAMBDA: return c->lambda;
    case OR_F_LAMBDAX: return c->lambdaX;
    case OR_F_LAMBDAY: return c->lambdaY;
    case OR_F_BROKEN: return c->broken;
    case OR_F_BREAKFORCE: return c->breakForce;
    case OR_F_FORCE: return c->force;
    case OR_F_TARGET: return c->target;
    case OR_F_REST: return c->rest;
    case OR_F_MINANGLE: return c->minAngle;
    case OR_F_MAXANGLE: return c->maxAngle;
    case OR_F_OWNER: return c->owner;
    case OR_F_COLOR: return c->color;
    default: return NAN;
  }
}

void or_con_set(or_world *w, int id, int field, double v) {
  orc_t *c = &w->cons[id];
  switch (field) {
    case OR_F_TYPE: c->type = (int)v; break;
    case OR_F_A: c->a = (int)v; break;
    case OR_F_B: c->b = (int)v; break;
    case OR_F_LAX: c->lax = v; break;
    case OR_F_LAY: c->lay = v; break;
    case OR_F_LBX: c->lbx = v; break;
    case OR_F_LBY: c->lby = v; break;
    case OR_F_COMPLIANCE: c->compliance = v; break;
    case OR_F_LAMBDA: c->lambda = v; break;
    case OR_F_LAMBDAX: c->lambdaX = v; break;
    case OR_F_LAMBDAY: c->lambdaY = v; break;
    case OR_F_BROKEN: c->broken = v != 0; break;
    case OR_F_BREAKFORCE: c->breakForce = v; break;
    case OR_F_FORCE: c->force = v; break;
    case OR_F_TARGET: c->target = v; break;
    case OR_F_REST: c->rest = v; break;
    case OR_F_MINANGLE: c->minAngle = v; break;
    case OR_F_MAXANGLE: c->maxAngle = v; break;
    case OR_F_OWNER: c->owner = (int)v; break;
    case OR_F_COLOR: c->color = (int)v; break;
    default: break;
  }
}

int or_world_list(const or_world *w, int k) { return w->list[k]; }
void or_world_set_list(or_world *w, const int *ids, int n) {
  if (n != w->nC) return;
  memcpy(w->list, ids, sizeof(int) * (size_t)n);
}

void or_world_set_rects(or_world *w, const double *rects, int n) {
  free(w->rects);
  w->rects = NULL;
  w->nR = n;
  w->hasSdf = 1;
  if (n > 0) {
    w->rects = (double *)malloc(sizeof(double) * 4 * (size_t)n);
    memcpy(w->rects, rects, sizeof(double) * 4 * (size_t)n);
  }
}

void or_world_color_info(const or_world *w, uint32_t *off16, uint32_t *cnt16) {
  memcpy(off16, w->colorOff, sizeof(w->colorOff));
  memcpy(cnt16, w->colorCnt, sizeof(w->colorCnt));
}

void or_world_stats(const or_world *w, double *maxSpeed, double *maxAngSpeed,
                    int *nan, long *collisions, int *broken) {
  *maxSpeed = w->st_maxSpeed;
  *maxAngSpeed = w->st_maxAngSpeed;
  *nan = w->st_nan;
  *collisions = w->st_collisions;
  *broken = w->st_broken;
}

/* ======================================================================
 * colouring: assignColor / ensureColored (xpbd.js:98-126),
 * groupConstraintsByColor (core.js:276-288)
 * ==================================================================== */
int or_assign_color(uint32_t *mask, int a, int b) {
  return or_assign_color_n(mask, 0x7fffffff, a, b);
}

/* assignColor over a mask of n entries with Uint32Array semantics: reads
 * past the end give 0, writes past the end are dropped (createSim's mask
 * has 1 << 16 entries, core.js:45) */
int or_assign_color_n(uint32_t *mask, int n, int a, int b) {
  uint32_t ma = a < n ? mask[a] : 0u;
  uint32_t mb = (b >= 0 && b < n) ? mask[b] : 0u;
  uint32_t used = ma | mb;
  int c = 0;
  while (c < 32 && (used & (1u << c))) c++;
  if (c >= 32) c = 31;
  if (a < n) mask[a] = ma | (1u << c);
  if (b >= 0 && b < n) mask[b] = mb | (1u << c);
  return c;
}

void or_group_by_color(or_world *w) {
  int *out = (int *)malloc(sizeof(int) * (size_t)(w->nC > 0 ? w->nC : 1));
  int n = 0;
  uint32_t maxCnt = 0;
  for (int col = 0; col < OR_MAX_COLORS; col++) {
    w->colorOff[col] = (uint32_t)n;
    uint32_t cnt = 0;
    for (int k = 0; k < w->nC; k++) {
      int id = w->list[k];
      if ((w->cons[id].color | 0) == col) { out[n++] = id; cnt++; }
    }
    w->colorCnt[col] = cnt;
    if (cnt > maxCnt) maxCnt = cnt;
  }
  memcpy(w->list, out, sizeof(int) * (size_t)n);
  free(out);
  w->colorMax = maxCnt;
  w->colored = 1;
}

void or_ensure_colored(or_world *w) {
  if (w->colored) return;
  size_t m = (size_t)(w->n * 2 > 1024 ? w->n * 2 : 1024);
  uint32_t *mask = (uint32_t *)calloc(m, sizeof(uint32_t));
  for (int k = 0; k < w->nC; k++) {
    orc_t *c = &w->cons[w->list[k]];
    if (c->color < 0) c->color = or_assign_color(mask, c->a, c->b >= 0 ? c->b : -1);
  }
  free(mask);
  or_group_by_color(w);
}

/* ======================================================================
 * map.js
 * ==================================================================== */
/* mulberry32, map.js:11-20 */
uint32_t or_mulberry32_next(uint32_t *state, double *out) {
  uint32_t a = *state + 0x6D2B79F5u;
  *state = a;
  uint32_t t = a;
  t = (t ^ (t >> 15)) * (t | 1u);
  t ^= t + (t ^ (t >> 7)) * (t | 61u);
  uint32_t r = t ^ (t >> 14);
  if (out) *out = (double)r / 4294967296.0;
  return r;
}

double or_rnd(uint32_t *state) {
  double v;
  or_mulberry32_next(state, &v);
  return v;
}

static void push_rect(double *out, int *n, int max, double x, double y, double w, double h) {
  if (*n < max) {
    out[4 * *n + 0] = x; out[4 * *n + 1] = y;
    out[4 * *n + 2] = w; out[4 * *n + 3] = h;
  }
  (*n)++;
}

/* makeMap rect list, map.js:22-59 (the lights that follow draw from the same
 * stream after every rect is placed, so they do not change the rects) */
int or_make_map(double width, double height, double T, int cols, int rows,
                double density, uint32_t seed, double *out, int max) {
  int n = 0;
  push_rect(out, &n, max, 0, 0, width, T);
  push_rect(out, &n, max, 0, height - T, width, T);
  push_rect(out, &n, max, 0, 0, T, height);
  push_rect(out, &n, max, width - T, 0, T, height);
  uint32_t rs = seed;
  double cw = width / cols, ch = height / rows;
  for (int col = 1; col < cols; col++) {
    double xl = col * cw;
    for (int row = 0; row < rows; row++) {
      if (or_rnd(&rs) > density) continue;
      double ys = row * ch;
      double gSz = fmax(60, fmin(ch * (0.28 + or_rnd(&rs) * 0.38), height * 0.4));
      double gStart = ys + or_rnd(&rs) * fmax(1, ch - gSz);
      double wt = 10 + floor(or_rnd(&rs) * 10);
      if (gStart > ys + 14) push_rect(out, &n, max, xl - wt / 2, ys, wt, gStart - ys);
      double gEnd = gStart + gSz;
      if (gEnd < ys + ch - 14) push_rect(out, &n, max, xl - wt / 2, gEnd, wt, ys + ch - gEnd);
    }
  }
  for (int row = 1; row < rows; row++) {
    double yl = row * ch;
    for (int col = 0; col < cols; col++) {
      if (or_rnd(&rs) > density) continue;
      double xs = col * cw;
      double gSz = fmax(60, fmin(cw * (0.28 + or_rnd(&rs) * 0.38), width * 0.3));
      double gStart = xs + or_rnd(&rs) * fmax(1, cw - gSz);
      double wt = 10 + floor(or_rnd(&rs) * 10);
      if (gStart > xs + 14) push_rect(out, &n, max, xs, yl - wt / 2, gStart - xs, wt);
      double gEnd = gStart + gSz;
      if (gEnd < xs + cw - 14) push_rect(out, &n, max, gEnd, yl - wt / 2, xs + cw - gEnd, wt);
    }
  }
  return n;
}

/* makeSdf, map.js:91-118. Returns 0 where the JS returns null. */
int or_sdf(const double *rects, int n, double x, double y, double *d, double *nx, double *ny) {
  double best = INFINITY, bnx = 0, bny = 0;
  for (int i = 0; i < n; i++) {
    const double *r = rects + 4 * i;
    double cx = fmax(r[0], fmin(x, r[0] + r[2]));
    double cy = fmax(r[1], fmin(y, r[1] + r[3]));
    double dx = x - cx, dy = y - cy;
    double d2 = dx * dx + dy * dy;
    if (d2 > 1e-12) {
      if (d2 < best * best) {
        double dd = sqrt(d2);
        best = dd; bnx = dx / dd; bny = dy / dd;
      }
    } else {
      double dl = x - r[0], dr = r[0] + r[2] - x, dt = y - r[1], db = r[1] + r[3] - y;
      double m = fmin(fmin(dl, dr), fmin(dt, db));
      double dd = -m;
      if (dd < best) {
        best = dd;
        if (m == dl) { bnx = -1; bny = 0; }
        else if (m == dr) { bnx = 1; bny = 0; }
        else if (m == dt) { bnx = 0; bny = -1; }
        else { bnx = 0; bny = 1; }
      }
    }
  }
  if (!isfinite(best)) return 0;
  *d = best; *nx = bnx; *ny = bny;
  return 1;
}

/* findSpawn, map.js:120-128 */
void or_find_spawn(const double *rects, int n, double width, double height,
                   double clearance, uint32_t *rng, double *ox, double *oy) {
  for (int i = 0; i < 500; i++) {
    double x = clearance + or_rnd(rng) * fmax(1, width - clearance * 2);
    double y = clearance + or_rnd(rng) * fmax(1, height - clearance * 2);
    double d, nx, ny;
    if (or_sdf(rects, n, x, y, &d, &nx, &ny) && d >= clearance) {
      *ox = x; *oy = y;
      return;
    }
  }
  *ox = width * 0.5;
  *oy = height * 0.5;
}

/* ======================================================================
 * ref64: XpbdWorld physics (xpbd.js)
 * ==================================================================== */
/* wrapAngle, xpbd.js:128-134 */
static double wrap_angle(double a) {
  const double TAU = JS_PI * 2;
  double d = fmod(a, TAU);
  if (d > JS_PI) d -= TAU;
  else if (d < -JS_PI) d += TAU;
  return d;
}

/* angleDelta, xpbd.js:137-143 */
static double angle_delta(double a, double b) {
  double d = fmod(a - b, JS_PI * 2);
  if (!isfinite(d)) return 0;
  if (d > JS_PI) d -= JS_PI * 2;
  else if (d < -JS_PI) d += JS_PI * 2;
  return d;
}

/* _solvePin, xpbd.js:331-389 */
static void solve_pin(or_world *w, orc_t *c, int firstIteration) {
  if (firstIteration) { c->lambdaX = 0; c->lambdaY = 0; }
  int A = c->a, B = c->b;
  double *ppx = PPX(w), *ppy = PPY(w), *angP = ANGP(w), *im = IM(w), *ii = II(w);
  double ca = cos(angP[A]), sa = sin(angP[A]);
  double rax = c->lax * ca - c->lay * sa, ray = c->lax * sa + c->lay * ca;
  double gax = ppx[A] + rax, gay = ppy[A] + ray;
  double gbx, gby, rbx = 0, rby = 0, wB = 0, wIB = 0;
  if (B >= 0) {
    double cb = cos(angP[B]), sb = sin(angP[B]);
    rbx = c->lbx * cb - c->lby * sb; rby = c->lbx * sb + c->lby * cb;
    gbx = ppx[B] + rbx; gby = ppy[B] + rby;
    wB = im[B]; wIB = ii[B];
  } else {
    gbx = c->lbx; gby = c->lby;
  }
  double Cx = gax - gbx, Cy = gay - gby;
  if (!isfinite(Cx) || !isfinite(Cy)) return;
  if (Cx * Cx + Cy * Cy < SLACK_POS * SLACK_POS) return;
  double pax = -ray, pay = rax;
  double pbx = -rby, pby = rbx;
  double wA = im[A], wIA = ii[A];
  double wSum = wA + wB;
  double k00 = wSum + wIA * pax * pax + wIB * pbx * pbx;
  double k01 = wIA * pax * pay + wIB * pbx * pby;
  double k11 = wSum + wIA * pay * pay + wIB * pby * pby;
  double det = k00 * k11 - k01 * k01;
  if (fabs(det) < 1e-12) return;
  double alphaTilde = c->compliance / (w->h * w->h);
  double bx = Cx + alphaTilde * c->lambdaX;
  double by = Cy + alphaTilde * c->lambdaY;
  double i00 = k11 / det, i11 = k00 / det, i01 = -k01 / det;
  double dlx = -(i00 * bx + i01 * by);
  double dly = -(i01 * bx + i11 * by);
  if (!isfinite(dlx) || !isfinite(dly)) return;
  c->lambdaX += dlx; c->lambdaY += dly;
  ppx[A] += wA * dlx; ppy[A] += wA * dly;
  angP[A] += wIA * (pax * dlx + pay * dly);
  if (B >= 0) {
    ppx[B] -= wB * dlx; ppy[B] -= wB * dly;
    angP[B] -= wIB * (pbx * dlx + pby * dly);
  }
}

/* _solveAngle, xpbd.js:392-439 */
static void solve_angle(or_world *w, orc_t *c, int firstIteration) {
  if (firstIteration) c->lambda = 0;
  int A = c->a, B = c->b;
  double *angP = ANGP(w), *ii = II(w);
  double wA = ii[A], wB = B >= 0 ? ii[B] : 0;
  double wSum = wA + wB;
  if (wSum <= 0) return;
  double rel = B >= 0 ? angle_delta(angP[B], angP[A]) : angP[A];
  double dev = angle_delta(rel, c->rest);
  double C = angle_delta(dev, c->target);
  if (!isfinite(C)) return;
  if (fabs(C) >= SLACK_ANG) {
    double alphaTilde = c->compliance / (w->h * w->h);
    double dl = -(C + alphaTilde * c->lambda) / (wSum + alphaTilde);
    if (!isfinite(dl)) return;
    c->lambda += dl;
    if (B >= 0) { angP[B] += wB * dl; angP[A] -= wA * dl; }
    else { angP[A] += wA * dl; }
  }
  double rel2 = B >= 0 ? angle_delta(angP[B], angP[A]) : angP[A];
  double dev2 = angle_delta(rel2, c->rest);
  double over = 0;
  if (dev2 > c->maxAngle) over = dev2 - c->maxAngle;
  else if (dev2 < c->minAngle) over = dev2 - c->minAngle;
  if (fabs(over) >= SLACK_ANG && wSum > 0) {
    double dl2 = -over / wSum;
    if (B >= 0) { angP[B] += wB * dl2; angP[A] -= wA * dl2; }
    else { angP[A] += wA * dl2; }
  }
}

/* _solveCollisions, xpbd.js:447-469 */
void or_solve_collisions(or_world *w) {
  if (!w->hasSdf) return;
  double *ppx = PPX(w), *ppy = PPY(w), *angP = ANGP(w), *im = IM(w);
  for (int k = 0; k < w->nP; k++) {
    int B = w->cpBody[k];
    double ca = cos(angP[B]), sa = sin(angP[B]);
    double wx = ppx[B] + w->cpLx[k] * ca - w->cpLy[k] * sa;
    double wy = ppy[B] + w->cpLx[k] * sa + w->cpLy[k] * ca;
    double d, nx, ny;
    if (!or_sdf(w->rects, w->nR, wx, wy, &d, &nx, &ny)) continue;
    double pen = w->cpR[k] - d;
    if (pen <= SLACK_POS) continue;
    if (im[B] == 0) continue;
    ppx[B] += nx * pen;
    ppy[B] += ny * pen;
    w->st_collisions++;
  }
}

/* _measure, xpbd.js:471-484 */
static void measure(or_world *w) {
  double mv = 0, mw = 0;
  int nan = 0;
  for (int i = 0; i < w->n; i++) {
    double s = hypot(VX(w)[i], VY(w)[i]);
    if (s > mv) mv = s;
    double a = fabs(AV(w)[i]);
    if (a > mw) mw = a;
    if (!isfinite(PX(w)[i]) || !isfinite(PY(w)[i]) || !isfinite(ANG(w)[i])) nan++;
  }
  w->st_maxSpeed = mv;
  w->st_maxAngSpeed = mw;
  w->st_nan = nan;
}

/* substep, xpbd.js:257-328 */
void or_substep(or_world *w) {
  const double h = w->h;
  const int n = w->n;
  double *px = PX(w), *py = PY(w), *ppx = PPX(w), *ppy = PPY(w), *vx = VX(w), *vy = VY(w);
  double *ang = ANG(w), *angP = ANGP(w), *av = AV(w), *im = IM(w), *ii = II(w);
  double *fx = FX(w), *fy = FY(w), *tq = TQ(w);
  double linDamp = exp(-w->linDrag * h);
  double angDamp = exp(-w->angDrag * h);
  for (int i = 0; i < n; i++) {
    if (im[i] == 0 && ii[i] == 0) {
      ppx[i] = px[i]; ppy[i] = py[i]; angP[i] = ang[i];
      vx[i] = 0; vy[i] = 0; av[i] = 0;
      continue;
    }
    vx[i] = (vx[i] + h * im[i] * fx[i]) * linDamp;
    vy[i] = (vy[i] + h * im[i] * fy[i]) * linDamp;
    av[i] = (av[i] + h * ii[i] * tq[i]) * angDamp;
    double sp = hypot(vx[i], vy[i]);
    if (sp > w->maxSpeed) { double k = w->maxSpeed / sp; vx[i] *= k; vy[i] *= k; }
    if (av[i] > w->maxAngSpeed) av[i] = w->maxAngSpeed;
    else if (av[i] < -w->maxAngSpeed) av[i] = -w->maxAngSpeed;
    if (!isfinite(vx[i]) || !isfinite(vy[i])) { vx[i] = 0; vy[i] = 0; w->st_nan++; }
    if (!isfinite(av[i])) { av[i] = 0; w->st_nan++; }
    ppx[i] = px[i] + h * vx[i];
    ppy[i] = py[i] + h * vy[i];
    angP[i] = ang[i] + h * av[i];
    fx[i] = 0; fy[i] = 0; tq[i] = 0;
  }
  for (int it = 0; it < w->iterations; it++) {
    for (int k = 0; k < w->nC; k++) {
      orc_t *c = &w->cons[w->list[k]];
      if (c->broken) continue;
      if (c->type == OR_C_ANGLE) solve_angle(w, c, it == 0);
      else solve_pin(w, c, it == 0);
    }
    or_solve_collisions(w);
  }
  for (int i = 0; i < n; i++) {
    vx[i] = (ppx[i] - px[i]) / h;
    vy[i] = (ppy[i] - py[i]) / h;
    av[i] = angle_delta(angP[i], ang[i]) / h;
    double sp2 = hypot(vx[i], vy[i]);
    if (sp2 > w->maxSpeed) { double k = w->maxSpeed / sp2; vx[i] *= k; vy[i] *= k; }
    if (av[i] > w->maxAngSpeed) av[i] = w->maxAngSpeed;
    else if (av[i] < -w->maxAngSpeed) av[i] = -w->maxAngSpeed;
    px[i] = ppx[i]; py[i] = ppy[i];
    ang[i] = angP[i];
    if (ang[i] > 50 || ang[i] < -50) { double wr = wrap_angle(ang[i]); ang[i] = wr; angP[i] = wr; }
  }
  measure(w);
}

/* _postGripBreak, xpbd.js:496-504 */
static void post_grip_break(or_world *w) {
  double inv = 1 / w->h;
  for (int k = 0; k < w->nC; k++) {
    orc_t *c = &w->cons[w->list[k]];
    if (c->type != OR_C_GRIP || c->broken) continue;
    double f = hypot(c->lambdaX, c->lambdaY) * inv;
    c->force = f;
    if (f > c->breakForce) { c->broken = 1; w->st_broken++; }
  }
}

/* step, xpbd.js:487-490 */
void or_step(or_world *w) {
  for (int s = 0; s < w->substeps; s++) or_substep(w);
  post_grip_break(w);
}

/* ======================================================================
 * ref32: f32solver.mjs (collMode 'seq')
 * ==================================================================== */
#ifdef OR_COUNT_OPS
static uint64_t g_ops;
#define OPC(k) (g_ops += (uint64_t)(k))
#else
#define OPC(k) ((void)0)
#endif
uint64_t or_f32_op_count(void) {
#ifdef OR_COUNT_OPS
  return g_ops;
#else
  return 0;
#endif
}
void or_f32_op_count_reset(void) {
#ifdef OR_COUNT_OPS
  g_ops = 0;
#endif
}

/* one rounding op each, like one f() call of f32solver.mjs */
static inline float f_add(float a, float b) { OPC(1); return a + b; }
static inline float f_sub(float a, float b) { OPC(1); return a - b; }
static inline float f_mul(float a, float b) { OPC(1); return a * b; }
static inline float f_div(float a, float b) { OPC(1); return a / b; }
static inline float f_sqrt(float a) { OPC(1); return sqrtf(a); }
static inline float f_cos(float a) { OPC(1); return (float)cos((double)a); }
static inline float f_sin(float a) { OPC(1); return (float)sin((double)a); }

static const float F_SLACK_POS = 0.002f;         /* f(0.002) */
static const float F_SLACK_ANG = 0.0002f;        /* f(0.0002) */
static const float F_TAU = 6.28318530718f;       /* f(6.28318530718) */
static const float F_PI = 3.14159265359f;        /* f(3.14159265359) */
static const float F_EPS_DET = 1e-12f;
static const float F_EPS_SDF = 1e-12f;
static const float F_SDF_INF = 1e30f;
static const float F_SDF_VALID = 1e29f;

/* WGSL `%` with FRem semantics; q from the f64 quotient, f32solver.mjs:36-51 */
static float angle_delta_f(float a, float b) {
  float x = f_sub(a, b);
  double q = trunc((double)x / (double)F_TAU);
  OPC(1);
  float d = f_sub(x, (float)((double)F_TAU * q));
  if (d > F_PI) return f_sub(d, F_TAU);
  if (d < -F_PI) return f_add(d, F_TAU);
  return d;
}

static float wrap_angle_f(float a) {
  double q = trunc((double)a / (double)F_TAU);
  OPC(1);
  float d = f_sub(a, (float)((double)F_TAU * q));
  if (d > F_PI) return f_sub(d, F_TAU);
  if (d < -F_PI) return f_add(d, F_TAU);
  return d;
}

/* WGSL length(vec2f), f32solver.mjs:54-56 */
static float length_f(float x, float y) { return f_sqrt(f_add(f_mul(x, x), f_mul(y, y))); }

/* f32ify statics, f32solver.mjs:63-112 */
void or_f32ify(or_world *w) {
  f32snap_t *f = &w->f;
  f32_free(f);
  f->active = 1;
  int n = w->n, nC = w->nC, nP = w->nP, nR = w->nR;
  f->n = n; f->nC = nC; f->nP = nP; f->nR = nR;
  f->h = (float)w->h;
  f->invH = (float)(1 / w->h);
  f->invH2 = (float)(1 / (w->h * w->h));
  float nl = -(float)w->linDrag, na = -(float)w->angDrag;
  f->linDamp = (float)exp((double)(nl * f->h));
  f->angDamp = (float)exp((double)(na * f->h));
  f->maxSpeed = (float)w->maxSpeed;
  f->maxAngSpeed = (float)w->maxAngSpeed;
  f->imF = (float *)malloc(sizeof(float) * (size_t)(n + 1));
  f->iiF = (float *)malloc(sizeof(float) * (size_t)(n + 1));
  for (int i = 0; i < n; i++) { f->imF[i] = (float)IM(w)[i]; f->iiF[i] = (float)II(w)[i]; }
  size_t cN = (size_t)(nC + 1);
  f->laxF = (float *)malloc(sizeof(float) * cN); f->layF = (float *)malloc(sizeof(float) * cN);
  f->restF = (float *)malloc(sizeof(float) * cN); f->minF = (float *)malloc(sizeof(float) * cN);
  f->maxF = (float *)malloc(sizeof(float) * cN);
  f->typeArr = (int *)malloc(sizeof(int) * cN); f->aArr = (int *)malloc(sizeof(int) * cN);
  f->bArr = (int *)malloc(sizeof(int) * cN); f->conId = (int *)malloc(sizeof(int) * cN);
  f->compF = (float *)malloc(sizeof(float) * cN); f->tgtF = (float *)malloc(sizeof(float) * cN);
  f->lbxF = (float *)malloc(sizeof(float) * cN); f->lbyF = (float *)malloc(sizeof(float) * cN);
  f->brkF = (float *)malloc(sizeof(float) * cN);
  for (int k = 0; k < nC; k++) {
    orc_t *c = &w->cons[w->list[k]];
    f->conId[k] = w->list[k];
    f->laxF[k] = (float)c->lax; f->layF[k] = (float)c->lay;
    f->restF[k] = (float)c->rest; f->minF[k] = (float)c->minAngle; f->maxF[k] = (float)c->maxAngle;
    f->typeArr[k] = c->type; f->aArr[k] = c->a; f->bArr[k] = c->b;
  }
  size_t rN = (size_t)(nR + 1);
  f->rx = (float *)malloc(sizeof(float) * rN); f->ry = (float *)malloc(sizeof(float) * rN);
  f->rxw = (float *)malloc(sizeof(float) * rN); f->ryh = (float *)malloc(sizeof(float) * rN);
  for (int i = 0; i < nR; i++) {
    const double *r = w->rects + 4 * i;
    f->rx[i] = (float)r[0]; f->ry[i] = (float)r[1];
    f->rxw[i] = (float)r[0] + (float)r[2];
    f->ryh[i] = (float)r[1] + (float)r[3];
  }
  size_t pN = (size_t)(nP + 1);
  f->cpBody = (int *)malloc(sizeof(int) * pN);
  f->cpLx = (float *)malloc(sizeof(float) * pN); f->cpLy = (float *)malloc(sizeof(float) * pN);
  f->cpR = (float *)malloc(sizeof(float) * pN);
  for (int i = 0; i < nP; i++) {
    f->cpBody[i] = w->cpBody[i];
    f->cpLx[i] = (float)w->cpLx[i]; f->cpLy[i] = (float)w->cpLy[i]; f->cpR[i] = (float)w->cpR[i];
  }
  /* bodyPts: points per body in collPts order, f32solver.mjs:314-315 */
  f->bpOff = (int *)calloc((size_t)(n + 1), sizeof(int));
  f->bpCnt = (int *)calloc((size_t)(n + 1), sizeof(int));
  f->bpIdx = (int *)malloc(sizeof(int) * pN);
  for (int i = 0; i < nP; i++) f->bpCnt[f->cpBody[i]]++;
  int acc = 0;
  for (int b = 0; b < n; b++) { f->bpOff[b] = acc; acc += f->bpCnt[b]; }
  int *cur = (int *)malloc(sizeof(int) * (size_t)(n + 1));
  memcpy(cur, f->bpOff, sizeof(int) * (size_t)n);
  for (int i = 0; i < nP; i++) f->bpIdx[cur[f->cpBody[i]]++] = i;
  free(cur);
}

/* roundState, f32solver.mjs:128-135 */
void or_f32_round_state(or_world *w) {
  for (int i = 0; i < w->n; i++) {
    PX(w)[i] = (float)PX(w)[i]; PY(w)[i] = (float)PY(w)[i];
    PPX(w)[i] = (float)PPX(w)[i]; PPY(w)[i] = (float)PPY(w)[i];
    VX(w)[i] = (float)VX(w)[i]; VY(w)[i] = (float)VY(w)[i];
    ANG(w)[i] = (float)ANG(w)[i]; ANGP(w)[i] = (float)ANGP(w)[i]; AV(w)[i] = (float)AV(w)[i];
  }
}

/* snapshotControls, f32solver.mjs:118-125 */
static void snapshot_controls(or_world *w) {
  f32snap_t *f = &w->f;
  for (int k = 0; k < f->nC; k++) {
    orc_t *c = &w->cons[f->conId[k]];
    f->compF[k] = (float)c->compliance; f->tgtF[k] = (float)c->target;
    f->lbxF[k] = (float)c->lbx; f->lbyF[k] = (float)c->lby;
    f->brkF[k] = (float)(isfinite(c->breakForce) ? fmin(c->breakForce, 1e30) : 1e30);
  }
}

/* sdfF, f32solver.mjs:139-166 */
static int sdf_f(const f32snap_t *f, float x, float y, float *od, float *onx, float *ony) {
  float best = F_SDF_INF, bnx = 0, bny = 0;
  for (int i = 0; i < f->nR; i++) {
    float cx = x < f->rx[i] ? f->rx[i] : (x > f->rxw[i] ? f->rxw[i] : x);
    float cy = y < f->ry[i] ? f->ry[i] : (y > f->ryh[i] ? f->ryh[i] : y);
    float dx = f_sub(x, cx), dy = f_sub(y, cy);
    float d2 = f_add(f_mul(dx, dx), f_mul(dy, dy));
    if (d2 > F_EPS_SDF) {
      if (d2 < f_mul(best, best)) {
        best = f_sqrt(d2);
        bnx = f_div(dx, best); bny = f_div(dy, best);
      }
    } else {
      float dl = f_sub(x, f->rx[i]), dr = f_sub(f->rxw[i], x);
      float dt = f_sub(y, f->ry[i]), db = f_sub(f->ryh[i], y);
      float m = dl, nx = -1, ny = 0;
      if (dr < m) { m = dr; nx = 1; ny = 0; }
      if (dt < m) { m = dt; nx = 0; ny = -1; }
      if (db < m) { m = db; nx = 0; ny = 1; }
      float d = -m;
      if (d < best) { best = d; bnx = nx; bny = ny; }
    }
  }
  if (best > F_SDF_VALID) return 0;
  *od = best; *onx = bnx; *ony = bny;
  return 1;
}

/* resetLambdaF, f32solver.mjs:169-174 */
static void reset_lambda_f(or_world *w) {
  for (int k = 0; k < w->nC; k++) {
    orc_t *c = &w->cons[w->list[k]];
    c->lambdaX = 0; c->lambdaY = 0; c->lambda = 0;
  }
}

/* integrateF, f32solver.mjs:177-200 */
static void integrate_f(or_world *w) {
  f32snap_t *f = &w->f;
  const float h = f->h;
  for (int i = 0; i < w->n; i++) {
    if (f->imF[i] == 0 && f->iiF[i] == 0) {
      PPX(w)[i] = PX(w)[i]; PPY(w)[i] = PY(w)[i]; ANGP(w)[i] = ANG(w)[i];
      VX(w)[i] = 0; VY(w)[i] = 0; AV(w)[i] = 0;
      continue;
    }
    float vx = f_mul(f_add((float)VX(w)[i], f_mul(f_mul(h, f->imF[i]), (float)FX(w)[i])), f->linDamp);
    float vy = f_mul(f_add((float)VY(w)[i], f_mul(f_mul(h, f->imF[i]), (float)FY(w)[i])), f->linDamp);
    float av = f_mul(f_add((float)AV(w)[i], f_mul(f_mul(h, f->iiF[i]), (float)TQ(w)[i])), f->angDamp);
    float sp = length_f(vx, vy);
    if (sp > f->maxSpeed) { float k = f_div(f->maxSpeed, sp); vx = f_mul(vx, k); vy = f_mul(vy, k); }
    if (av > f->maxAngSpeed) av = f->maxAngSpeed;
    else if (av < -f->maxAngSpeed) av = -f->maxAngSpeed;
    if (!(vx == vx) || !(vy == vy)) { vx = 0; vy = 0; }
    if (!(av == av)) av = 0;
    VX(w)[i] = vx; VY(w)[i] = vy; AV(w)[i] = av;
    PPX(w)[i] = f_add((float)PX(w)[i], f_mul(h, vx));
    PPY(w)[i] = f_add((float)PY(w)[i], f_mul(h, vy));
    ANGP(w)[i] = f_add((float)ANG(w)[i], f_mul(h, av));
    FX(w)[i] = 0; FY(w)[i] = 0; TQ(w)[i] = 0;
  }
}

/* solvePinF, f32solver.mjs:203-256 */
static void solve_pin_f(or_world *w, int k) {
  f32snap_t *f = &w->f;
  orc_t *c = &w->cons[f->conId[k]];
  double *ppx = PPX(w), *ppy = PPY(w), *angP = ANGP(w);
  int A = f->aArr[k];
  float ca = f_cos((float)angP[A]), sa = f_sin((float)angP[A]);
  float rax = f_sub(f_mul(f->laxF[k], ca), f_mul(f->layF[k], sa));
  float ray = f_add(f_mul(f->laxF[k], sa), f_mul(f->layF[k], ca));
  float gax = f_add((float)ppx[A], rax), gay = f_add((float)ppy[A], ray);
  float gbx = f->lbxF[k], gby = f->lbyF[k];
  float rbx = 0, rby = 0, wB = 0, wIB = 0;
  int B = f->bArr[k];
  if (B >= 0) {
    float cb = f_cos((float)angP[B]), sb = f_sin((float)angP[B]);
    rbx = f_sub(f_mul(f->lbxF[k], cb), f_mul(f->lbyF[k], sb));
    rby = f_add(f_mul(f->lbxF[k], sb), f_mul(f->lbyF[k], cb));
    gbx = f_add((float)ppx[B], rbx); gby = f_add((float)ppy[B], rby);
    wB = f->imF[B]; wIB = f->iiF[B];
  }
  float Cx = f_sub(gax, gbx), Cy = f_sub(gay, gby);
  if (!(Cx == Cx) || !(Cy == Cy)) return;
  if (f_add(f_mul(Cx, Cx), f_mul(Cy, Cy)) < f_mul(F_SLACK_POS, F_SLACK_POS)) return;
  float pax = -ray, pay = rax;
  float pbx = -rby, pby = rbx;
  float wA = f->imF[A], wIA = f->iiF[A];
  float wSum = f_add(wA, wB);
  float k00 = f_add(f_add(wSum, f_mul(f_mul(wIA, pax), pax)), f_mul(f_mul(wIB, pbx), pbx));
  float k01 = f_add(f_mul(f_mul(wIA, pax), pay), f_mul(f_mul(wIB, pbx), pby));
  float k11 = f_add(f_add(wSum, f_mul(f_mul(wIA, pay), pay)), f_mul(f_mul(wIB, pby), pby));
  float det = f_sub(f_mul(k00, k11), f_mul(k01, k01));
  if (fabsf(det) < F_EPS_DET) return;
  float alphaTilde = f_mul(f->compF[k], f->invH2);
  float bx = f_add(Cx, f_mul(alphaTilde, (float)c->lambdaX));
  float by = f_add(Cy, f_mul(alphaTilde, (float)c->lambdaY));
  float i00 = f_div(k11, det), i11 = f_div(k00, det), i01 = -f_div(k01, det);
  float dlx = -f_add(f_mul(i00, bx), f_mul(i01, by));
  float dly = -f_add(f_mul(i01, bx), f_mul(i11, by));
  if (!(dlx == dlx) || !(dly == dly)) return;
  c->lambdaX = f_add((float)c->lambdaX, dlx);
  c->lambdaY = f_add((float)c->lambdaY, dly);
  ppx[A] = f_add((float)ppx[A], f_mul(wA, dlx));
  ppy[A] = f_add((float)ppy[A], f_mul(wA, dly));
  angP[A] = f_add((float)angP[A], f_mul(wIA, f_add(f_mul(pax, dlx), f_mul(pay, dly))));
  if (B >= 0) {
    ppx[B] = f_sub((float)ppx[B], f_mul(wB, dlx));
    ppy[B] = f_sub((float)ppy[B], f_mul(wB, dly));
    angP[B] = f_sub((float)angP[B], f_mul(wIB, f_add(f_mul(pbx, dlx), f_mul(pby, dly))));
  }
}

/* solveAngleF, f32solver.mjs:258-301 */
static void solve_angle_f(or_world *w, int k) {
  f32snap_t *f = &w->f;
  orc_t *c = &w->cons[f->conId[k]];
  double *angP = ANGP(w);
  int A = f->aArr[k], B = f->bArr[k];
  int hasB = B >= 0;
  float wA = f->iiF[A];
  float wB = 0;
  float rel = (float)angP[A];
  if (hasB) { wB = f->iiF[B]; rel = angle_delta_f((float)angP[B], (float)angP[A]); }
  float wSum = f_add(wA, wB);
  if (wSum <= 0) return;
  float dev = angle_delta_f(rel, f->restF[k]);
  float C = angle_delta_f(dev, f->tgtF[k]);
  if (!(C == C)) return;
  if (fabsf(C) >= F_SLACK_ANG) {
    float alphaTilde = f_mul(f->compF[k], f->invH2);
    float dl = -f_div(f_add(C, f_mul(alphaTilde, (float)c->lambda)), f_add(wSum, alphaTilde));
    if (!(dl == dl)) return;
    c->lambda = f_add((float)c->lambda, dl);
    if (hasB) {
      angP[B] = f_add((float)angP[B], f_mul(wB, dl));
      angP[A] = f_sub((float)angP[A], f_mul(wA, dl));
    } else {
      angP[A] = f_add((float)angP[A], f_mul(wA, dl));
    }
  }
  float rel2 = (float)angP[A];
  if (hasB) rel2 = angle_delta_f((float)angP[B], (float)angP[A]);
  float dev2 = angle_delta_f(rel2, f->restF[k]);
  float over = 0;
  if (dev2 > f->maxF[k]) over = f_sub(dev2, f->maxF[k]);
  else if (dev2 < f->minF[k]) over = f_sub(dev2, f->minF[k]);
  if (fabsf(over) >= F_SLACK_ANG) {
    float dl2 = -f_div(over, wSum);
    if (hasB) {
      angP[B] = f_add((float)angP[B], f_mul(wB, dl2));
      angP[A] = f_sub((float)angP[A], f_mul(wA, dl2));
    } else {
      angP[A] = f_add((float)angP[A], f_mul(wA, dl2));
    }
  }
}

/* solveConstraintsF, f32solver.mjs:303-310 */
static void solve_constraints_f(or_world *w) {
  f32snap_t *f = &w->f;
  for (int k = 0; k < f->nC; k++) {
    orc_t *c = &w->cons[f->conId[k]];
    if (c->broken) continue;
    if (f->typeArr[k] == OR_C_ANGLE) solve_angle_f(w, k);
    else solve_pin_f(w, k);
  }
}

/* solveCollisionsF 'seq' + pointDelta, f32solver.mjs:317-344 */
static void solve_collisions_f(or_world *w) {
  f32snap_t *f = &w->f;
  double *ppx = PPX(w), *ppy = PPY(w), *angP = ANGP(w);
  for (int b = 0; b < w->n; b++) {
    for (int q = 0; q < f->bpCnt[b]; q++) {
      int i = f->bpIdx[f->bpOff[b] + q];
      if (f->imF[b] == 0) continue;
      float ca = f_cos((float)angP[b]), sa = f_sin((float)angP[b]);
      float wx = f_add((float)ppx[b], f_sub(f_mul(f->cpLx[i], ca), f_mul(f->cpLy[i], sa)));
      float wy = f_add((float)ppy[b], f_add(f_mul(f->cpLx[i], sa), f_mul(f->cpLy[i], ca)));
      float d, nx, ny;
      if (!sdf_f(f, wx, wy, &d, &nx, &ny)) continue;
      float pen = f_sub(f->cpR[i], d);
      if (pen <= F_SLACK_POS) continue;
      ppx[b] = f_add((float)ppx[b], f_mul(nx, pen));
      ppy[b] = f_add((float)ppy[b], f_mul(ny, pen));
      w->st_collisions++;
    }
  }
}

/* finalizeF, f32solver.mjs:376-399 */
static void finalize_f(or_world *w) {
  f32snap_t *f = &w->f;
  for (int i = 0; i < w->n; i++) {
    if (f->imF[i] == 0 && f->iiF[i] == 0) {
      VX(w)[i] = 0; VY(w)[i] = 0; AV(w)[i] = 0;
      continue;
    }
    float vx = f_mul(f_sub((float)PPX(w)[i], (float)PX(w)[i]), f->invH);
    float vy = f_mul(f_sub((float)PPY(w)[i], (float)PY(w)[i]), f->invH);
    float av = f_mul(angle_delta_f((float)ANGP(w)[i], (float)ANG(w)[i]), f->invH);
    float sp = length_f(vx, vy);
    if (sp > f->maxSpeed) { float k = f_div(f->maxSpeed, sp); vx = f_mul(vx, k); vy = f_mul(vy, k); }
    if (av > f->maxAngSpeed) av = f->maxAngSpeed;
    else if (av < -f->maxAngSpeed) av = -f->maxAngSpeed;
    VX(w)[i] = vx; VY(w)[i] = vy; AV(w)[i] = av;
    PX(w)[i] = PPX(w)[i]; PY(w)[i] = PPY(w)[i];
    ANG(w)[i] = ANGP(w)[i];
    if (ANG(w)[i] > 50 || ANG(w)[i] < -50) {
      float wr = wrap_angle_f((float)ANG(w)[i]);
      ANG(w)[i] = wr; ANGP(w)[i] = wr;
    }
  }
}

/* gripBreakF, f32solver.mjs:402-416 */
static void grip_break_f(or_world *w) {
  f32snap_t *f = &w->f;
  double invH64 = 1 / w->h;
  for (int k = 0; k < f->nC; k++) {
    orc_t *c = &w->cons[f->conId[k]];
    if (f->typeArr[k] != OR_C_GRIP || c->broken) continue;
    float fm = f_mul(length_f((float)c->lambdaX, (float)c->lambdaY), f->invH);
    if (fm > f->brkF[k]) {
      c->broken = 1; c->lambdaX = 0; c->lambdaY = 0;
      c->force = 0;
      w->st_broken++;
    } else {
      c->force = hypot(c->lambdaX, c->lambdaY) * invH64;
    }
  }
}

/* patched substep/step, f32solver.mjs:419-434 */
static void substep_f(or_world *w) {
  reset_lambda_f(w);
  integrate_f(w);
  for (int it = 0; it < w->iterations; it++) {
    solve_constraints_f(w);
    solve_collisions_f(w);
  }
  finalize_f(w);
  measure(w);
}

void or_step32(or_world *w) {
  if (!w->f.active) or_f32ify(w);
  snapshot_controls(w);
  for (int s = 0; s < w->substeps; s++) substep_f(w);
  grip_break_f(w);
}

/* ======================================================================
 * kraken.js
 * ==================================================================== */
double or_arm_reach(int segs) { return B_SHOULDER_R + segs * B_SEGLEN; } /* kraken.js:49 */

static double rect_inertia(double m, double w, double h) { return m * (w * w + h * h) / 12; }

/* spawnKraken, kraken.js:64-148, with BODY.arms / BODY.segsPerArm as arguments */
int or_spawn_kraken(or_world *w, double x, double y, double angle, int arms, int segs,
                    double curl, or_kraken *out) {
  if (arms < 1 || arms > OR_MAX_ARMS || segs < 1 || segs > OR_MAX_SEGS) return -1;
  memset(out, 0, sizeof(*out));
  out->nArms = arms; out->nSegs = segs;
  double mantleI = (B_MANTLE_MASS * B_MANTLE_R * B_MANTLE_R / 2) * B_MANTLE_IF;
  int mantle = or_add_body(w, x, y, angle, B_MANTLE_MASS, mantleI);
  out->mantle = mantle;
  for (int i = 0; i < 8; i++) {
    double a = ((double)i / 8) * JS_PI * 2;
    or_add_collision_point(w, mantle, cos(a) * B_MANTLE_R * 0.7, sin(a) * B_MANTLE_R * 0.7,
                           B_MANTLE_R * 0.45);
  }
  for (int a = 0; a < arms; a++) {
    double relAng = ((double)a / arms) * JS_PI * 2;
    double th0 = angle + relAng;
    double jx = x + cos(th0) * B_SHOULDER_R;
    double jy = y + sin(th0) * B_SHOULDER_R;
    double th = th0;
    for (int i = 0; i < segs; i++) {
      double t = segs > 1 ? (double)i / (segs - 1) : 0;
      double mass = B_SEG_MASS_PROX + (B_SEG_MASS_DIST - B_SEG_MASS_PROX) * t;
      double thick = B_SEG_THICK_PROX + (B_SEG_THICK_DIST - B_SEG_THICK_PROX) * t;
      double ux = cos(th), uy = sin(th);
      double cx = jx + ux * B_SEGLEN * 0.5;
      double cy = jy + uy * B_SEGLEN * 0.5;
      int b = or_add_body(w, cx, cy, th, mass, rect_inertia(mass, B_SEGLEN, thick));
      double r = thick * 0.5;
      or_add_collision_point(w, b, -B_SEGLEN * 0.5 + r * 0.4, 0, r);
      or_add_collision_point(w, b, B_SEGLEN * 0.5 - r * 0.4, 0, r);
      out->segs[a][i] = b;
      jx = cx + ux * B_SEGLEN * 0.5;
      jy = cy + uy * B_SEGLEN * 0.5;
      th += curl;
    }
    or_add_constraint(w, OR_C_PIN, mantle, out->segs[a][0], cos(relAng) * B_SHOULDER_R,
                      sin(relAng) * B_SHOULDER_R, -B_SEGLEN * 0.5, 0, 0);
    int ms = or_add_constraint(w, OR_C_ANGLE, mantle, out->segs[a][0], 0, 0, 0, 0, 1 / B_STIFF_MIN);
    w->cons[ms].rest = relAng;
    w->cons[ms].target = 0;
    w->cons[ms].minAngle = -shoulder_limit();
    w->cons[ms].maxAngle = shoulder_limit();
    w->cons[ms].owner = a;
    out->motors[a][0] = ms;
    for (int i = 0; i < segs - 1; i++) {
      or_add_constraint(w, OR_C_PIN, out->segs[a][i], out->segs[a][i + 1], B_SEGLEN * 0.5, 0,
                        -B_SEGLEN * 0.5, 0, 0);
      int m = or_add_constraint(w, OR_C_ANGLE, out->segs[a][i], out->segs[a][i + 1], 0, 0, 0, 0,
                                1 / B_STIFF_MIN);
      w->cons[m].rest = curl;
      w->cons[m].target = 0;
      w->cons[m].minAngle = -joint_limit();
      w->cons[m].maxAngle = joint_limit();
      w->cons[m].owner = a;
      out->motors[a][i + 1] = m;
    }
    int tip = out->segs[a][segs - 1];
    int g = or_add_constraint(w, OR_C_GRIP, tip, -1, B_SEGLEN * 0.5, 0, x, y, 0);
    w->cons[g].broken = 1;
    w->cons[g].breakForce = 0;
    w->cons[g].owner = a;
    out->grip[a] = g;
    out->tip[a] = tip;
    out->relAng[a] = relAng;
  }
  out->spawnX = x; out->spawnY = y; out->spawnAngle = angle;
  return mantle;
}

/* tipPosition, kraken.js:150-154 */
void or_tip_position(const or_world *w, const or_kraken *k, int arm, double *x, double *y) {
  int b = k->tip[arm];
  double L = B_SEGLEN * 0.5;
  double c = cos(w->arr[OR_A_ANG][b]), s = sin(w->arr[OR_A_ANG][b]);
  *x = w->arr[OR_A_PX][b] + L * c;
  *y = w->arr[OR_A_PY][b] + L * s;
}

/* attachGrip, kraken.js:157-164 */
void or_attach_grip(or_world *w, const or_kraken *k, int arm, double breakForce) {
  double tx, ty;
  or_tip_position(w, k, arm, &tx, &ty);
  orc_t *g = &w->cons[k->grip[arm]];
  g->lbx = tx; g->lby = ty;
  g->broken = 0;
  g->breakForce = breakForce;
  g->lambdaX = 0; g->lambdaY = 0; g->force = 0;
}

/* releaseGrip, kraken.js:166 */
void or_release_grip(or_world *w, const or_kraken *k, int arm) {
  orc_t *g = &w->cons[k->grip[arm]];
  g->broken = 1;
  g->force = 0;
}

/* toneToCompliance, kraken.js:186-191 */
double or_tone_to_compliance(double tone) {
  double t = fmax(0, fmin(1, tone));
  double stiff = B_STIFF_MIN + t * (B_STIFF_MAX - B_STIFF_MIN);
  return 1 / stiff;
}

/* adhesionToBreakForce, kraken.js:194-198 */
double or_adhesion_to_break_force(double a) {
  double c = fmax(0, fmin(1, a));
  return B_GRIP_MIN + (B_GRIP_MAX - B_GRIP_MIN) * c;
}

/* ======================================================================
 * core.js: createSim, applyControl, readProprio
 * ==================================================================== */
typedef struct {
  or_kraken k;
  double tone;
  double adhesion[OR_MAX_ARMS], cd[OR_MAX_ARMS];
  double prevVx, prevVy;
  or_metrics m;
  double sx, sy;                       /* preStep's position */
  int armWasAnchored[OR_MAX_ARMS], wasAnchored;
} or_creature;

struct or_sim {
  or_world *w;
  double width, height;
  int nR;
  double *rects;
  int nCr;
  or_creature *cr;
  double gripSlipMax, gripCooldown;
};

/* An empty sim on the given map (rects x y w h), solver constants of
 * XpbdWorld's defaults with the given substeps / iterations / h. */
or_sim *or_sim_new(double width, double height, const double *rects, int nR, int substeps,
                   int iterations, double h) {
  or_sim *s = (or_sim *)calloc(1, sizeof(or_sim));
  s->w = or_world_new(substeps, iterations, h, 3.0, 3.0, 360, 18);
  s->width = width; s->height = height;
  s->gripSlipMax = 150;
  s->gripCooldown = 0.05;
  s->nR = nR;
  s->rects = (double *)malloc(sizeof(double) * 4 * (size_t)(nR > 0 ? nR : 1));
  if (nR > 0) memcpy(s->rects, rects, sizeof(double) * 4 * (size_t)nR);
  or_world_set_rects(s->w, s->rects, s->nR);
  return s;
}

/* Adds one creature at a given pose (spawnKraken, kraken.js:64-148) with its
 * constraints coloured in creation order on a fresh per-creature mask (the
 * colours createSim gives a creature whose bodies are all below 65536) and
 * the whole list regrouped by colour; returns the creature index. */
int or_sim_add_creature(or_sim *s, double x, double y, double angle, int arms, int segs) {
  int c0 = s->w->nC;
  s->cr = (or_creature *)realloc(s->cr, sizeof(or_creature) * (size_t)(s->nCr + 1));
  or_creature *c = &s->cr[s->nCr];
  memset(c, 0, sizeof(*c));
  if (or_spawn_kraken(s->w, x, y, angle, arms, segs, B_SPAWN_CURL, &c->k) < 0) return -1;
  c->tone = 0.5;
  uint32_t *mask = (uint32_t *)calloc((size_t)s->w->n, sizeof(uint32_t));
  for (int id = c0; id < s->w->nC; id++) {
    orc_t *cc = &s->w->cons[id];
    if (cc->color < 0) cc->color = or_assign_color(mask, cc->a, cc->b >= 0 ? cc->b : -1);
  }
  free(mask);
  s->w->colored = 0;
  or_group_by_color(s->w);
  return s->nCr++;
}

/* createSim, core.js:37-74 (prey 0; senses, lights and fitness are not on
 * the physics path). Colouring follows core.js:45-58: one body mask for the
 * whole world, constraints coloured in creation order, then grouped. */
or_sim *or_sim_create(uint32_t seed, int creatures, double width, double height,
                      int substeps, int iterations, double h, int arms, int segs) {
  double tmp[4 * 256];
  int nR = or_make_map(width, height, 14, 4, 3, 0.48, seed, tmp, 256);
  if (nR > 256) nR = 256;
  or_sim *s = or_sim_new(width, height, tmp, nR, substeps, iterations, h);
  uint32_t rnd = seed ^ 0x9e3779b9u;
  s->nCr = creatures;
  s->cr = (or_creature *)calloc((size_t)(creatures > 0 ? creatures : 1), sizeof(or_creature));
  uint32_t *mask = (uint32_t *)calloc(1u << 16, sizeof(uint32_t));
  for (int i = 0; i < creatures; i++) {
    double x, y;
    or_find_spawn(s->rects, s->nR, width, height, or_arm_reach(segs) + 20, &rnd, &x, &y);
    double ang = or_rnd(&rnd) * JS_PI * 2;
    or_spawn_kraken(s->w, x, y, ang, arms, segs, B_SPAWN_CURL, &s->cr[i].k);
    for (int id = 0; id < s->w->nC; id++) {
      orc_t *c = &s->w->cons[id];
      if (c->color < 0) c->color = or_assign_color_n(mask, 1 << 16, c->a, c->b >= 0 ? c->b : -1);
    }
    s->cr[i].tone = 0.5;
  }
  free(mask);
  or_group_by_color(s->w);
  return s;
}

void or_sim_free(or_sim *s) {
  if (!s) return;
  or_world_free(s->w);
  free(s->rects);
  free(s->cr);
  free(s);
}

or_world *or_sim_world(or_sim *s) { return s->w; }
int or_sim_rects(const or_sim *s, double *out, int max) {
  int n = s->nR < max ? s->nR : max;
  memcpy(out, s->rects, sizeof(double) * 4 * (size_t)n);
  return s->nR;
}
int or_sim_ncreatures(const or_sim *s) { return s->nCr; }
void or_sim_kraken(const or_sim *s, int i, or_kraken *out) { *out = s->cr[i].k; }
void or_sim_set_reflex(or_sim *s, double gripSlipMax, double gripCooldown) {
  s->gripSlipMax = gripSlipMax;
  s->gripCooldown = gripCooldown;
}
void or_sim_reflex_state(const or_sim *s, int ci, double *cd, double *adhesion) {
  const or_creature *c = &s->cr[ci];
  for (int a = 0; a < c->k.nArms; a++) { cd[a] = c->cd[a]; adhesion[a] = c->adhesion[a]; }
}

/* the suction-cup reflex of applyControl, core.js:199-218 */
static void reflex(or_sim *s, or_creature *c, int a, double adhesionCtl) {
  or_world *w = s->w;
  double adh = fmax(0, fmin(1, adhesionCtl));
  c->adhesion[a] = adh;
  if (c->cd[a] > 0) c->cd[a] -= w->h * w->substeps;
  orc_t *g = &w->cons[c->k.grip[a]];
  if (g->broken) {
    if (adh > 0.08 && c->cd[a] <= 0) {
      int tip = c->k.tip[a];
      double slip = hypot(VX(w)[tip], VY(w)[tip]);
      if (slip < s->gripSlipMax) or_attach_grip(w, &c->k, a, or_adhesion_to_break_force(adh));
      else c->cd[a] = s->gripCooldown;
    }
  } else {
    g->breakForce = or_adhesion_to_break_force(adh);
    if (adh < 0.04) or_release_grip(w, &c->k, a);
  }
}

/* applyControl, core.js:183-220 */
void or_apply_control(or_sim *s, int ci, double tone, const double *shoulder,
                      const double *curl, const double *adhesion) {
  or_creature *c = &s->cr[ci];
  or_world *w = s->w;
  c->tone = fmax(0, fmin(1, tone));
  double comp = or_tone_to_compliance(c->tone);
  for (int a = 0; a < c->k.nArms; a++) {
    for (int j = 0; j < c->k.nSegs; j++) w->cons[c->k.motors[a][j]].compliance = comp;
    w->cons[c->k.motors[a][0]].target = fmax(-shoulder_limit(), fmin(shoulder_limit(), shoulder[a]));
    for (int j = 1; j < c->k.nSegs; j++)
      w->cons[c->k.motors[a][j]].target = fmax(-joint_limit(), fmin(joint_limit(), curl[a]));
    reflex(s, c, a, adhesion[a]);
  }
}

/* applyControl with one commanded deviation per motor instead of the
 * shoulder + shared curl pair (core.js:195-198 clamps each the same way) */
void or_apply_control_motors(or_sim *s, int ci, double tone, const double *targets,
                             const double *adhesion) {
  or_creature *c = &s->cr[ci];
  or_world *w = s->w;
  c->tone = fmax(0, fmin(1, tone));
  double comp = or_tone_to_compliance(c->tone);
  int S = c->k.nSegs;
  for (int a = 0; a < c->k.nArms; a++) {
    for (int j = 0; j < S; j++) w->cons[c->k.motors[a][j]].compliance = comp;
    w->cons[c->k.motors[a][0]].target =
        fmax(-shoulder_limit(), fmin(shoulder_limit(), targets[a * S]));
    for (int j = 1; j < S; j++)
      w->cons[c->k.motors[a][j]].target =
          fmax(-joint_limit(), fmin(joint_limit(), targets[a * S + j]));
    reflex(s, c, a, adhesion[a]);
  }
}

/* armCurl, kraken.js:169-176 */
static double arm_curl(const or_world *w, const or_kraken *k, int a) {
  double sum = 0;
  int n = 0;
  for (int i = 1; i < k->nSegs; i++) {
    double d = w->arr[OR_A_ANG][k->segs[a][i]] - w->arr[OR_A_ANG][k->segs[a][i - 1]];
    sum += atan2(sin(d), cos(d));
    n++;
  }
  return n ? sum / n : 0;
}

/* armExtension, kraken.js:179-183 */
static double arm_extension(const or_world *w, const or_kraken *k, int a) {
  double tx, ty;
  or_tip_position(w, k, a, &tx, &ty);
  int s0 = k->segs[a][0];
  double reach = or_arm_reach(k->nSegs);
  return fmin(1, hypot(tx - w->arr[OR_A_PX][s0], ty - w->arr[OR_A_PY][s0]) / fmax(1, reach));
}

static double clamp_sym(double v, double m) { return v > m ? m : (v < -m ? -m : v); }

/* readProprio, core.js:129-175 (6 values per arm + 6 body values) */
int or_read_proprio(or_sim *s, int ci, double *out) {
  or_creature *c = &s->cr[ci];
  or_world *w = s->w;
  const or_kraken *k = &c->k;
  int m = k->mantle, A = k->nArms;
  double cx = PX(w)[m], cy = PY(w)[m], cvx = VX(w)[m], cvy = VY(w)[m];
  double angle = ANG(w)[m], cav = AV(w)[m];
  double speed = hypot(cvx, cvy);
  double ca = cos(-angle), sa = sin(-angle);
  int anchored = 0;
  double extSum = 0, curlSum = 0;
  double shoulder[OR_MAX_ARMS];
  double reach = or_arm_reach(k->nSegs);
  for (int a = 0; a < A; a++) {
    double d = ANG(w)[k->segs[a][0]] - angle;
    shoulder[a] = atan2(sin(d), cos(d));
    extSum += arm_extension(w, k, a);
    curlSum += arm_curl(w, k, a);
    if (!w->cons[k->grip[a]].broken) anchored++;
  }
  int i = 0;
  for (int a = 0; a < A; a++) out[i++] = clamp_sym(shoulder[a] / shoulder_limit(), 1.2);
  for (int a = 0; a < A; a++) out[i++] = clamp_sym(arm_curl(w, k, a) / joint_limit(), 1.2);
  for (int a = 0; a < A; a++) {
    double tx, ty;
    or_tip_position(w, k, a, &tx, &ty);
    double dx = tx - cx, dy = ty - cy;
    out[i++] = clamp_sym((dx * ca - dy * sa) / reach, 1.2);
    out[i++] = clamp_sym((dx * sa + dy * ca) / reach, 1.2);
  }
  for (int a = 0; a < A; a++) {
    const orc_t *g = &w->cons[k->grip[a]];
    double fo = g->force == g->force ? g->force : 0; /* (g.force || 0) */
    out[i++] = g->broken ? 0 : fmin(1, fo / fmax(1, g->breakForce));
  }
  for (int a = 0; a < A; a++) out[i++] = w->cons[k->grip[a]].broken ? 0 : 1;
  double ax = (cvx - c->prevVx) / (w->h * w->substeps);
  double ay = (cvy - c->prevVy) / (w->h * w->substeps);
  out[i++] = fmax(-1, fmin(1, (ax * ca - ay * sa) / 600));
  out[i++] = fmax(-1, fmin(1, (ax * sa + ay * ca) / 600));
  c->prevVx = cvx; c->prevVy = cvy;
  out[i++] = (double)anchored / A;
  out[i++] = extSum / A;
  out[i++] = fmin(1, speed / 300);
  out[i++] = fmax(-1, fmin(1, cav / 18));
  return i;
}

void or_sim_step(or_sim *s) { or_step(s->w); }

/* measureReach, fitness.js:74-88: the free space around (x, y) along 16
 * rays marched in 12 px steps up to 3.5 arm reaches, until the SDF of the
 * map is not positive */
double or_measure_reach(const double *rects, int nR, double reach, double x, double y) {
  double sum = 0, best = 0;
  const int N = 16;
  for (int k = 0; k < N; k++) {
    const double a = ((double)k / N) * JS_PI * 2;
    double d = 0;
    while (d < reach * 3.5) {
      d += 12;
      double hd, nx, ny;
      if (!or_sdf(rects, nR, x + cos(a) * d, y + sin(a) * d, &hd, &nx, &ny) || hd <= 0) break;
    }
    sum += d;
    if (d > best) best = d;
  }
  const double r = (sum / N) * 0.55 + best * 0.45;
  return r > 70 ? r : 70;
}

void or_sim_set_spawn_reach(or_sim *s, int ci, double reach) { s->cr[ci].m.spawnReach = reach; }

/* preStep, core.js:291-294 */
void or_sim_pre_step(or_sim *s) {
  for (int i = 0; i < s->nCr; i++) {
    or_creature *c = &s->cr[i];
    c->sx = PX(s->w)[c->k.mantle];
    c->sy = PY(s->w)[c->k.mantle];
  }
}

/* postStep, core.js:297-356 (no prey) */
void or_sim_post_step(or_sim *s) {
  const or_world *w = s->w;
  for (int i = 0; i < s->nCr; i++) {
    or_creature *c = &s->cr[i];
    or_metrics *m = &c->m;
    const int mt = c->k.mantle, A = c->k.nArms;
    const double x = PX(w)[mt], y = PY(w)[mt], angle = ANG(w)[mt], av = AV(w)[mt];
    m->steps++;
    const double dx = x - c->sx, dy = y - c->sy;
    const double stepDist = hypot(dx, dy);
    m->pathLen += stepDist;
    m->angularAccum += fabs(av) * w->h * w->substeps;
    const double fa = angle - JS_PI * 0.5;
    const double fwd = dx * cos(fa) + dy * sin(fa);
    if (fwd > 0) m->forwardProg += fwd;
    int anchored = 0;
    for (int a = 0; a < A; a++) anchored += w->cons[c->k.grip[a]].broken ? 0 : 1;
    const double dSpawn = hypot(x - c->k.spawnX, y - c->k.spawnY);
    if (anchored > 0) {
      m->anchoredSteps++;
      if (dSpawn > m->spawnDistMax) { m->gripPullProg += dSpawn - m->spawnDistMax; m->spawnDistMax = dSpawn; }
    }
    if (anchored == 0 && stepDist > 0.3) m->freeMove += stepDist;
    m->energySpent += (c->tone * 0.0006 + stepDist * 0.0004) * A;
    if (anchored > 0 && !c->wasAnchored) m->gripCycles++;
    c->wasAnchored = anchored > 0;
    int newly = 0;
    for (int a = 0; a < A; a++) {
      const int now = w->cons[c->k.grip[a]].broken ? 0 : 1;
      if (now && !c->armWasAnchored[a]) { newly++; m->attachEvents++; }
      c->armWasAnchored[a] = now;
    }
    if (newly > 0 && anchored - newly > 0) m->strides += newly;
    if (dSpawn > m->maxDisplacement) m->maxDisplacement = dSpawn;
    m->x = x; m->y = y;
  }
}

/* score, fitness.js:115-172: the terms in TERM_ORDER, summed in f64 in that
 * order (no prey: preyHit and preyNear are 0); maxAngSpeed 18, dt 1/60 */
double or_score(const or_metrics *c) {
  const double W_gripPull = 2.6, W_strideBonus = 0.5, W_strideCap = 60, W_reach = 320, W_directed = 70,
               W_headingHold = 28, W_meanSpeed = 14, W_efficiency = 3, W_progGateKnee = 0.25, W_spin = 0.55,
               W_drift = 0.05, W_energy = 0.30;
  const double steps = c->steps > 1 ? c->steps : 1;
  const double path = c->pathLen, disp = c->maxDisplacement;
  const double reach = c->spawnReach > 0 ? c->spawnReach : 300;
  const double reachFrac = fmin(1.2, disp / reach);
  const double directed = path > 1 ? fmin(1, disp / path) : 0;
  const double spinBudget = steps * 18 * (1.0 / 60);
  const double headingHold = 1 - fmin(1, c->angularAccum / fmax(1e-6, spinBudget));
  const double meanSpeed = path / steps / 60;
  const double efficiency = c->forwardProg / fmax(0.5, c->energySpent > 0 ? c->energySpent : 0.5);
  const double progressBase = c->gripPullProg * W_gripPull + reachFrac * W_reach;
  const double strideFrac = fmin(c->strides, W_strideCap) / W_strideCap;
  const double progGate = fmin(1, disp / fmax(1e-6, W_progGateKnee * reach));
  const double t[12] = {
    c->gripPullProg * W_gripPull,
    progressBase * W_strideBonus * strideFrac,
    reachFrac * W_reach,
    directed * W_directed * progGate,
    headingHold * W_headingHold * progGate,
    fmin(1, meanSpeed) * W_meanSpeed * progGate,
    fmin(20, efficiency) * W_efficiency * progGate,
    -(c->angularAccum * W_spin * 0.02),
    -(c->freeMove * W_drift),
    -(c->energySpent * W_energy),
    0.0,
    0.0,
  };
  double sc = 0;
  for (int i = 0; i < 12; i++) sc += t[i];
  return isfinite(sc) ? sc : 0;
}

void or_sim_metrics(const or_sim *s, int ci, or_metrics *out) {
  *out = s->cr[ci].m;
  out->score = or_score(out);
}
void or_sim_step32(or_sim *s) { or_step32(s->w); }

/* ======================================================================
 * The trainer's controller: senses without entities (src/senses/echo.js,
 * light.js; tip contact core.js:260-266), the recurrent net (src/brain/
 * net.js:71-133) and one training step (src/sim/train.js:233-249 with
 * stepSim, core.js:358-382).  A sim's creatures share its time and lights.
 * ==================================================================== */
#define OR_ECHO_RAYS 12
#define OR_ECHO_RANGE 340.0
#define OR_SOUND_SPEED 900.0
#define OR_ECHO_INTERVAL 0.42
#define OR_MAX_LIGHTS 8
#define OR_NET_H 24
#define OR_NET_IN_MAX 128
#define OR_NET_OUT_MAX 32

typedef struct { double at; int i; double dist, intensity; } or_echo_pending;

typedef struct {
  double cooldown, range_[OR_ECHO_RAYS], intensity[OR_ECHO_RAYS];
  or_echo_pending pend[64];
  int npend, emitCount, wantsEmit;
  double light_l, light_r, light_t;
  double contact[OR_MAX_ARMS];
  float x[OR_NET_IN_MAX], h[2 * OR_NET_H], out[OR_NET_OUT_MAX];
} or_senses;

struct or_net_sim {
  or_sim *s;          /* borrowed */
  double time;
  int nL;
  double L[OR_MAX_LIGHTS][6];  /* x y r ir ph sp; x, y move */
  or_senses *cs;
  int n;
};
typedef struct or_net_sim or_net_sim;

/* a fresh trainer state for every creature of s and the map's lights */
or_net_sim *or_net_new(or_sim *s, const double *lights, int nL) {
  if (nL < 0 || nL > OR_MAX_LIGHTS) return NULL;
  or_net_sim *n = (or_net_sim *)calloc(1, sizeof(or_net_sim));
  n->s = s;
  n->nL = nL;
  for (int l = 0; l < nL; l++)
    for (int k = 0; k < 6; k++) n->L[l][k] = lights[6 * l + k];
  n->n = s->nCr;
  n->cs = (or_senses *)calloc((size_t)(s->nCr > 0 ? s->nCr : 1), sizeof(or_senses));
  return n;
}

void or_net_free(or_net_sim *n) {
  if (!n) return;
  free(n->cs);
  free(n);
}

int or_net_param_count(int arms) {
  const int ni = 10 * arms + 45, no = 3 * arms + 2, H = OR_NET_H;
  return ni * H + H + H * H + H + H * no + no;
}

/* forwardInto, net.js:71-98: f64 sums of the Float32Array's values,
 * activations stored back to f32; the second layer reads its bias at
 * b2 + j as the reference does */
static float net_act(double s) { return (float)(s > 20 ? 1 : (s < -20 ? -1 : tanh(s))); }

void or_net_forward(const float *w, const float *x, float *out, float *scratch, int nIn, int nOut) {
  const int H = OR_NET_H, h1 = 0, h2 = H;
  const int b1 = nIn * H, b2 = b1 + H, b3 = b2 + H * H, b4 = b3 + H, b5 = b4 + H * nOut;
  for (int j = 0; j < H; j++) {
    double s = w[b1 + j];
    const int row = j * nIn;
    for (int i = 0; i < nIn; i++) s += (double)x[i] * (double)w[row + i];
    scratch[h1 + j] = net_act(s);
  }
  for (int j = 0; j < H; j++) {
    double s = w[b2 + j];
    const int row = b3 - H * H + j * H;
    for (int i = 0; i < H; i++) s += (double)scratch[h1 + i] * (double)w[row + i];
    scratch[h2 + j] = net_act(s);
  }
  for (int j = 0; j < nOut; j++) {
    double s = w[b5 + j];
    const int row = b4 + j * H;
    for (int i = 0; i < H; i++) s += (double)scratch[h2 + i] * (double)w[row + i];
    out[j] = net_act(s);
  }
}

/* raymarch, echo.js:94-110 */
static double echo_raymarch(const or_sim *s, double x, double y, double angle, double maxDist) {
  const double dx = cos(angle), dy = sin(angle);
  double t = 0;
  for (int i = 0; i < 96; i++) {
    if (t >= maxDist) return maxDist;
    double d, nx, ny;
    if (!or_sdf(s->rects, s->nR, x + dx * t, y + dy * t, &d, &nx, &ny)) return maxDist;
    if (d <= 0) return t;
    t += fmax(1, d * 0.85);
    if (d < 0.5) return t;
  }
  return maxDist;
}

/* sampleAt, light.js:99-106 */
static double light_sample(const or_net_sim *n, double x, double y) {
  double v = 0.05;
  for (int l = 0; l < n->nL; l++) {
    const double d = hypot(x - n->L[l][0], y - n->L[l][1]);
    v += fmax(0, 1 - d / n->L[l][2]) * n->L[l][3];
  }
  return fmin(1, v);
}

/* tickSenses, core.js:245-267, with no entities */
static void tick_senses(or_net_sim *n, int ci) {
  or_sim *s = n->s;
  or_world *w = s->w;
  or_creature *c = &s->cr[ci];
  or_senses *e = &n->cs[ci];
  const int m = c->k.mantle;
  const double x = PX(w)[m], y = PY(w)[m], angle = ANG(w)[m];
  const double dt = w->h * w->substeps, time = n->time;
  const double heading = angle - JS_PI * 0.5;
  /* tick, echo.js:120-127 */
  if (e->cooldown > 0) e->cooldown -= dt;
  while (e->npend && e->pend[0].at <= time) {
    const or_echo_pending p = e->pend[0];
    memmove(e->pend, e->pend + 1, sizeof(or_echo_pending) * (size_t)(e->npend - 1));
    e->npend--;
    e->range_[p.i] = p.dist / OR_ECHO_RANGE;
    e->intensity[p.i] = p.intensity;
  }
  /* emit, echo.js:67-85 */
  if (e->wantsEmit && !(e->cooldown > 0)) {
    e->cooldown = OR_ECHO_INTERVAL;
    e->emitCount++;
    for (int i = 0; i < OR_ECHO_RAYS; i++) {
      const double t = (double)i / (OR_ECHO_RAYS - 1);
      const double a = heading + (t - 0.5) * (JS_PI * 0.85);
      const double d = echo_raymarch(s, x, y, a, OR_ECHO_RANGE);
      if (d >= OR_ECHO_RANGE) continue;
      const double inten = fmin(1, (OR_ECHO_RANGE * 0.22) / fmax(8, d * d / OR_ECHO_RANGE));
      if (e->npend < 64) {
        or_echo_pending p = {time + (2 * d) / OR_SOUND_SPEED, i, d, inten};
        e->pend[e->npend++] = p;
      }
    }
    /* the stable sort by arrival time */
    for (int a = 1; a < e->npend; a++) {
      const or_echo_pending p = e->pend[a];
      int b = a;
      while (b > 0 && e->pend[b - 1].at > p.at) { e->pend[b] = e->pend[b - 1]; b--; }
      e->pend[b] = p;
    }
    e->wantsEmit = 0;
  }
  /* sample, light.js:90-97 */
  const double perp = heading + JS_PI / 2;
  e->light_l = light_sample(n, x + cos(perp) * 26, y + sin(perp) * 26);
  e->light_r = light_sample(n, x - cos(perp) * 26, y - sin(perp) * 26);
  e->light_t = light_sample(n, x, y);
  /* tip contact, core.js:260-266 */
  for (int a = 0; a < c->k.nArms; a++) {
    double tx, ty, d, nx, ny;
    or_tip_position(w, &c->k, a, &tx, &ty);
    const double near = or_sdf(s->rects, s->nR, tx, ty, &d, &nx, &ny) ? fmax(0, 1 - d / 9) : 0;
    e->contact[a] = e->contact[a] * 0.7 + near * 0.3;
  }
}

/* One trainStep (train.js:233-249): per creature readProprio, readSenses,
 * the previous outputs, forwardInto with genome genomes[ind[ci]] (n_params
 * floats each), decode (net.js:124-133) and applyControl; then preStep, the
 * physics step (f32 emulation when f32, else f64), postStep, time, the
 * lights (tickMapLights, map.js:75-83) and tickSenses.  Returns -1 when a
 * creature's genome has the wrong size. */
int or_net_step(or_net_sim *n, const float *genomes, int n_params, const int *ind, int f32) {
  or_sim *s = n->s;
  or_world *w = s->w;
  for (int ci = 0; ci < s->nCr && ci < n->n; ci++) {
    or_creature *c = &s->cr[ci];
    or_senses *e = &n->cs[ci];
    const int A = c->k.nArms, no = 3 * A + 2;
    if (or_net_param_count(A) != n_params) return -1;
    double p[6 * OR_MAX_ARMS + 6];
    const int np = or_read_proprio(s, ci, p);
    int i = 0;
    for (int k = 0; k < np; k++) e->x[i++] = (float)p[k];
    for (int r = 0; r < OR_ECHO_RAYS; r++) {
      e->x[i++] = (float)e->range_[r];
      e->x[i++] = (float)e->intensity[r];
    }
    for (int k = 0; k < 6; k++) e->x[i++] = 0.f;  /* chemoreception: no scent sources */
    e->x[i++] = (float)e->light_l;
    e->x[i++] = (float)e->light_r;
    e->x[i++] = (float)e->light_t;
    for (int k = 0; k < 4; k++) e->x[i++] = 0.f;  /* hearing: no noise sources */
    for (int a = 0; a < A; a++) e->x[i++] = (float)e->contact[a];
    for (int k = 0; k < no; k++) e->x[i++] = e->out[k];
    or_net_forward(genomes + (size_t)ind[ci] * n_params, e->x, e->out, e->h, i, no);
    double shoulder[OR_MAX_ARMS], curl[OR_MAX_ARMS], adh[OR_MAX_ARMS];
    for (int a = 0; a < A; a++) {
      shoulder[a] = e->out[1 + 3 * a];
      curl[a] = e->out[2 + 3 * a];
      adh[a] = e->out[3 + 3 * a] > 0 ? e->out[3 + 3 * a] : 0;
    }
    e->wantsEmit = e->out[no - 1] > 0.3;
    or_apply_control(s, ci, 0.5 + 0.5 * e->out[0], shoulder, curl, adh);
  }
  or_sim_pre_step(s);
  if (f32) or_step32(w); else or_step(w);
  or_sim_post_step(s);
  const double dt = w->h * w->substeps;
  n->time += dt;
  for (int l = 0; l < n->nL; l++) {
    const double a = n->time * n->L[l][5] + n->L[l][4];
    n->L[l][0] = fmax(60, fmin(s->width - 60, n->L[l][0] + cos(a) * 18 * dt));
    n->L[l][1] = fmax(60, fmin(s->height - 60, n->L[l][1] + sin(a * 0.8) * 18 * dt));
  }
  for (int ci = 0; ci < s->nCr && ci < n->n; ci++) tick_senses(n, ci);
  return 0;
}

/* the last input vector and outputs of creature ci (n_in and n_out values) */
void or_net_io(const or_net_sim *n, int ci, float *x, float *out) {
  const int A = n->s->cr[ci].k.nArms;
  memcpy(x, n->cs[ci].x, sizeof(float) * (size_t)(10 * A + 45));
  memcpy(out, n->cs[ci].out, sizeof(float) * (size_t)(3 * A + 2));
}

/* echo state of creature ci: emissions so far and pending echoes */
void or_net_echo(const or_net_sim *n, int ci, int *emits, int *pending) {
  *emits = n->cs[ci].emitCount;
  *pending = n->cs[ci].npend;
}
