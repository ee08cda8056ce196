// kr_batch.cu -- the batched creature engine (include/kraken_batch.h).
//
// Work unit: a group of creatures of one body template.  A CTA of W warps
// takes a group from a device queue and stages the template's static arrays
// once in shared memory; every creature is advanced by G lanes of one warp
// (G = 32, 16 or 8, so a warp carries 32 / G creatures) for the whole run (up
// to max_steps env steps) with its state in shared memory and registers.
// Shared memory is carved per template: a CTA has a fixed budget, and a group
// holds as many creatures of its template as fit (at most W * 32 / G), so
// small bodies pack more creatures per CTA than large ones.  Groups are
// queued longest-remaining-horizon first so the tail of a run is short.  Per
// env step a creature's lanes compute the proprioception of the current state
// (f64, lanes over arms), draw or read the controls, run the suction-cup
// reflex (f64, lane per arm), then the XPBD step of kr_solver.cuh (f32 in
// f32solver.mjs op order) and the grip break.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "kr_batch_impl.h"
#include "kr_order.h"

namespace {
using namespace krb;

constexpr double kPiD = 3.141592653589793;
constexpr double kSegHalf = 13.5 * 0.5;                        // tipPosition L

struct BatchArgs {
  kr::SolverConsts K;
  const TplDev *tpl;
  TplArrays T;
  float *state;          // capacity x kStateStride
  float4 *grip;          // capacity x 8: lbx lby brk broken
  float2 *glam;          // capacity x 8: grip lambda after the last substep
  double2 *cd;           // capacity x 8: reflex cooldown, break force (f64, as applyControl sets it)
  float *ctrl_cur;       // capacity x kCtrlStride: the controls in use
  SlotMeta *meta;
  const float4 *rects;   // x y x+w y+h
  const int *map_off;    // n_maps + 1
  const float *map_cull; // per map cull distance
  const int *groups;     // n_groups x cpc slot ids, -1 = empty
  int n_groups;
  int cpc;               // creature entries per group (W * 32 / G)
  int *queue;            // group counter
  int max_steps;
  // Preemption (the rollout server's slices; null otherwise): once the word
  // turns non-zero, CTAs take no further group and every running creature
  // stops at its next env-step boundary, its state written back as after
  // any launch.  Each creature's lane 0 loads the word one step ahead, so
  // the load never stalls a step.
  const int *stop;
  // the rollout server's completion counts (null otherwise): a creature
  // that reaches its horizon adds 1 to tag_done[its SlotMeta::pad]
  int *tag_done;
  int ctrl_period;
  float *obs;            // capacity x ring x KR_OBS_STRIDE
  int obs_ring;
  double slip_max, cooldown, inv_h64, dt, h64;
  int substeps;
  // policy (KR_CTRL_POLICY: device layout, see policy(); KR_CTRL_NET: net.js layout)
  const float *pw;       // n_individuals x pw_stride
  const int *pw_idx;     // individual of each slot
  int pw_stride;
  // KR_CTRL_NET
  NetRec *net;           // capacity records
  const double *rects64; // x y w h per rect, f64 of the f32 values (offsets map_off)
  const double *lights;  // x y r ir ph sp per light
  const int *light_off;  // n_maps + 1, or null: no lights
  const double *map_size;
  const double2 *light_tab;  // per light, its position after env step t < light_T (or null)
  int light_T;
};

// --- shared-memory layout, carved per template ------------------------------
// Every region is a multiple of 4 words, so each region and each creature's
// base stay 16-byte aligned (the f64 and float4 views included).
constexpr int kLvlWords = (kr::kMaxTplLevels + 1 + 3) & ~3;                 // 68
constexpr int kArmWords = (3 * KR_BATCH_MAX_ARMS + KR_BATCH_MAX_ARMS * KR_BATCH_MAX_SEGS + 3) & ~3;
__host__ __device__ constexpr int r4(int n) { return (n + 3) & ~3; }

// statics of the template, once per CTA
__host__ __device__ inline int tpl_smem_words(int nb, int nc, int np) {
  return 5 * r4(nb) + 11 * r4(nc) + 4 * r4(np) + kLvlWords + kArmWords;
}
// one creature: the committed state (positions, angles, velocities: loaded
// from the slot's HBM block when the creature starts, written back when its
// run ends), predicted bodies and their sin/cos, grip and motor state,
// lambda, collision scratch
__host__ __device__ inline int creature_smem_words(int nb, int nc, int np, int arms, int segs) {
  return 11 * r4(nb) + 2 * r4(nc) + r4(arms * segs) + r4(arms * segs + arms) + 4 * arms + 3 * r4(np) +
         kr::kMaxCulled / 2;
}

struct TplSmem {
  float *im, *ii, *zero;
  int *boff, *bcnt, *ab, *type, *motor, *garm;
  float *lax, *lay, *lbx, *lby, *rest, *minA, *maxA;
  int *lvl;
  float *plx, *ply, *pr;
  int *pbody;
  int *arm_tip, *arm_grip, *arm_seg0, *arm_segs;
};

__device__ inline void carve_tpl(TplSmem &P, float *p, const TplDev &td) {
  const int mb = r4(td.nb), mc = r4(td.nc), mp = r4(td.np);
  P.im = p; p += mb; P.ii = p; p += mb; P.zero = p; p += mb;
  P.boff = reinterpret_cast<int *>(p); p += mb;
  P.bcnt = reinterpret_cast<int *>(p); p += mb;
  P.ab = reinterpret_cast<int *>(p); p += mc;
  P.type = reinterpret_cast<int *>(p); p += mc;
  P.motor = reinterpret_cast<int *>(p); p += mc;
  P.garm = reinterpret_cast<int *>(p); p += mc;
  P.lax = p; p += mc; P.lay = p; p += mc; P.lbx = p; p += mc; P.lby = p; p += mc;
  P.rest = p; p += mc; P.minA = p; p += mc; P.maxA = p; p += mc;
  P.lvl = reinterpret_cast<int *>(p); p += kLvlWords;
  P.plx = p; p += mp; P.ply = p; p += mp; P.pr = p; p += mp;
  P.pbody = reinterpret_cast<int *>(p); p += mp;
  P.arm_tip = reinterpret_cast<int *>(p); p += KR_BATCH_MAX_ARMS;
  P.arm_grip = reinterpret_cast<int *>(p); p += KR_BATCH_MAX_ARMS;
  P.arm_seg0 = reinterpret_cast<int *>(p); p += KR_BATCH_MAX_ARMS;
  P.arm_segs = reinterpret_cast<int *>(p);
}

struct CreatureSmem {
  float *ctrl;     // arms * segs motor controls, then arms adhesion values
  float *obs;      // proprioception (aliases the collision scratch pdy)
  double *pair;    // atan2 terms of armCurl (aliases the collision scratch pdx)
};

__device__ inline void carve_creature(kr::Island &S, CreatureSmem &X, const TplSmem &P, float *p,
                                      const TplDev &td) {
  const int mb = r4(td.nb), mc = r4(td.nc), mp = r4(td.np), AS = td.arms * td.segs;
  // committed state, resident for the creature's whole run
  S.px = p; p += mb; S.py = p; p += mb; S.vx = p; p += mb; S.vy = p; p += mb;
  S.ang = p; p += mb; S.av = p; p += mb;
  S.ppx = p; p += mb; S.ppy = p; p += mb; S.angP = p; p += mb;
  S.bs = p; p += mb; S.bc = p; p += mb;
  S.lamX = p; p += mc; S.lamY = p; p += mc;
  S.lam = S.lamX;  // pins use lamX/lamY, angles lam: never both on one slot
  S.tgt_m = p; p += r4(AS);
  X.ctrl = p; p += r4(AS + td.arms);
  S.anc = p; p += 4 * td.arms;
  S.pdx = p; p += mp; S.pdy = p; p += mp;
  S.pflag = reinterpret_cast<int *>(p); p += mp;
  S.cull = reinterpret_cast<short *>(p);
  // proprioception scratch: live only before the XPBD step of an env step,
  // when the collision scratch is dead (2 * arms * (segs - 1) <= np and
  // 6 * arms + 6 <= np for every template shape)
  X.pair = reinterpret_cast<double *>(S.pdx);
  X.obs = S.pdy;
  // statics shared by the CTA
  S.im = P.im; S.ii = P.ii; S.fx = P.zero; S.fy = P.zero; S.tq = P.zero;
  S.ab = P.ab; S.type = P.type; S.garm = P.garm; S.motor = P.motor;
  S.lax = P.lax; S.lay = P.lay; S.lbx = P.lbx; S.lby = P.lby;
  S.rest = P.rest; S.minA = P.minA; S.maxA = P.maxA;
  S.plx = P.plx; S.ply = P.ply; S.pr = P.pr; S.pbody = P.pbody; S.boff = P.boff; S.bcnt = P.bcnt;
  S.lvl = P.lvl;
  S.tb = nullptr; S.comp = nullptr; S.tgt = nullptr; S.brk = nullptr;
  S.nb = td.nb; S.nc = td.nc; S.np = td.np;
}

// mulberry32 (src/world/map.js:11-20): the draw is a hash of the state, and
// the state only advances by a constant, so the d-th draw after state s
// (d = 1, 2, ...) is mulberry_at(s + d * kMulberryStep): lanes draw their
// share of a redraw at once.
constexpr uint32_t kMulberryStep = 0x6D2B79F5u;
__device__ inline double mulberry_at(uint32_t t) {
  t = (t ^ (t >> 15)) * (t | 1u);
  t ^= t + (t ^ (t >> 7)) * (t | 61u);
  return (double)(t ^ (t >> 14)) / 4294967296.0;
}

__device__ inline double clamp_sym(double v, double m) { return v > m ? m : (v < -m ? -m : v); }

// One out-of-line copy of each f64 libm function that the reflex, postStep's
// accumulators, the proprioception, the net and the senses call (the same
// functions, with the same results): their call sites are many, and inlined
// at every one they made the NET kernel's per-step code larger than the
// instruction caches hold -- fetch stalls were its largest stall reason.
__device__ __noinline__ double2 lib_sincos(double x) {
  double s, c;
  sincos(x, &s, &c);
  return make_double2(s, c);
}
__device__ __noinline__ double lib_sin(double x) { return sin(x); }
__device__ __noinline__ double lib_cos(double x) { return cos(x); }
__device__ __noinline__ double lib_hypot(double x, double y) { return hypot(x, y); }
__device__ __noinline__ double lib_tanh(double x) { return tanh(x); }
__device__ __noinline__ double lib_atan2(double y, double x) { return atan2(y, x); }

// Math.atan2(Math.sin(d), Math.cos(d)) (kraken.js:173 armCurl, core.js:138
// the shoulder angle) for the f64 difference d of two angles, as the exact
// value that chain of f64 calls approximates to within a few ulp: d wrapped
// into (-pi, pi].  For |d| <= pi that is d itself;
// otherwise d - 2 pi k with k = rint(d / 2 pi) and 2 pi in three parts
// (k times each of the first two exact for |k| < 2^24, d - k p1 exact by
// Sterbenz), moved by one period more when the rounded quotient left the
// remainder outside [-pi, pi].  Beyond |d| = 2^20, and for non-finite d,
// the chain itself is evaluated.
__device__ __forceinline__ double wrap_pi(double d) {
  if (fabs(d) <= kPiD) return d;
  if (!(fabs(d) <= 1048576.0)) {
    const double2 sc = lib_sincos(d);
    return lib_atan2(sc.x, sc.y);
  }
  auto rem = [d](double k) {
    double r = fma(-k, 0x1.921fb54000000p+2, d);
    r = fma(-k, 0x1.10b4611000000p-28, r);
    return fma(-k, 0x1.4c4c6628b80dcp-57, r);
  };
  const double k = rint(d * 0.15915494309189535);  // 1 / (2 pi)
  double r = rem(k);
  if (r > kPiD) r = rem(k + 1);
  else if (r < -kPiD) r = rem(k - 1);
  return r;
}

// proprioception of the current state, readProprio (core.js:129-175), f64;
// writes 6A+6 values into X.obs and returns the attached-arm bitmask.  The
// grip load divides by the arm's break force in f64, cdp[a].y (the JS
// object's breakForce, which the GPU mirror never overwrites with the f32
// copy the solver holds).
template <int G>
__device__ unsigned proprio(const BatchArgs &A, const TplDev &td, const TplSmem &P, kr::Island &S,
                            CreatureSmem &X, SlotMeta &m, const double2 *cdp, const kr::Lanes<G> &L) {
  const int arms = td.arms, segs = td.segs, lane = L.lane;
  const float4 *grip_st = reinterpret_cast<const float4 *>(S.anc);
  const double cx = S.px[0], cy = S.py[0], cvx = S.vx[0], cvy = S.vy[0];
  const double angle = S.ang[0], cav = S.av[0];
  // armCurl terms: atan2(sin d, cos d) per adjacent segment pair, as wrap_pi
  const int npair = arms * (segs - 1);
  for (int q = lane; q < npair; q += G) {
    const int a = q / (segs - 1), i = q % (segs - 1) + 1;
    const double d = (double)S.ang[P.arm_segs[a * segs + i]] - (double)S.ang[P.arm_segs[a * segs + i - 1]];
    X.pair[q] = wrap_pi(d);
  }
  L.sync();
  double ext = 0.0, curl = 0.0, sh = 0.0, tx = 0.0, ty = 0.0;
  bool attached = false;
  if (lane < arms) {
    const int a = lane;
    double s = 0.0;
    for (int i = 0; i < segs - 1; i++) s += X.pair[a * (segs - 1) + i];
    curl = segs > 1 ? s / (segs - 1) : 0.0;
    const int s0 = P.arm_seg0[a], tip = P.arm_tip[a];
    const double d = (double)S.ang[s0] - angle;
    sh = wrap_pi(d);
    const double2 t = lib_sincos((double)S.ang[tip]);
    tx = (double)S.px[tip] + kSegHalf * t.y;
    ty = (double)S.py[tip] + kSegHalf * t.x;
    ext = fmin(1.0, lib_hypot(tx - (double)S.px[s0], ty - (double)S.py[s0]) / fmax(1.0, td.reach));
    attached = grip_st[a].w == 0.f;
  }
  const unsigned att = L.ballot(attached) & ((1u << arms) - 1u);
  // sums in arm order, like the sequential loop
  double ext_sum = 0.0;
  for (int a = 0; a < arms; a++) ext_sum += __shfl_sync(L.mask, ext, a, G);
  const double2 na = lib_sincos(-angle);
  const double sa = na.x, ca = na.y;
  const double SL = kPiD * 0.62, JL = kPiD * 0.42;
  if (lane < arms) {
    const int a = lane;
    X.obs[a] = (float)clamp_sym(sh / SL, 1.2);
    X.obs[arms + a] = (float)clamp_sym(curl / JL, 1.2);
    const double dx = tx - cx, dy = ty - cy;
    X.obs[2 * arms + 2 * a] = (float)clamp_sym((dx * ca - dy * sa) / td.reach, 1.2);
    X.obs[2 * arms + 2 * a + 1] = (float)clamp_sym((dx * sa + dy * ca) / td.reach, 1.2);
    const float4 g = grip_st[a];
    double force = 0.0;
    if (g.w == 0.f) force = lib_hypot((double)S.lamX[P.arm_grip[a]], (double)S.lamY[P.arm_grip[a]]) * A.inv_h64;
    X.obs[4 * arms + a] = g.w != 0.f ? 0.f : (float)fmin(1.0, force / fmax(1.0, cdp[a].y));
    X.obs[5 * arms + a] = g.w != 0.f ? 0.f : 1.f;
  }
  if (lane == 0) {
    const double ax = (cvx - m.prev_vx) / A.dt, ay = (cvy - m.prev_vy) / A.dt;
    X.obs[6 * arms] = (float)fmax(-1.0, fmin(1.0, (ax * ca - ay * sa) / 600));
    X.obs[6 * arms + 1] = (float)fmax(-1.0, fmin(1.0, (ax * sa + ay * ca) / 600));
    m.prev_vx = cvx;
    m.prev_vy = cvy;
    X.obs[6 * arms + 2] = (float)((double)__popc(att) / arms);
    X.obs[6 * arms + 3] = (float)(ext_sum / arms);
    X.obs[6 * arms + 4] = (float)fmin(1.0, lib_hypot(cvx, cvy) / 300);
    X.obs[6 * arms + 5] = (float)fmax(-1.0, fmin(1.0, cav / 18));
  }
  L.sync();
  return att;
}

// HPL consecutive floats from 8- or 16-byte aligned memory
template <int HPL>
__device__ __forceinline__ void load_vec(const float *p, float *v) {
  if constexpr (HPL == 2) {
    const float2 a = __ldg(reinterpret_cast<const float2 *>(p));
    v[0] = a.x; v[1] = a.y;
  } else {
#pragma unroll
    for (int k = 0; k < HPL; k += 4) {
      const float4 a = __ldg(reinterpret_cast<const float4 *>(p + k));
      v[k] = a.x; v[k + 1] = a.y; v[k + 2] = a.z; v[k + 3] = a.w;
    }
  }
}

// fused policy (G lanes): proprio (n_in = 6A + 6) -> 64 tanh -> A*S motor
// targets (tanh) + A adhesion values ((tanh + 1) / 2).  Device layout of an
// individual (the transpose of the public row-major layout, so lanes read
// consecutive words): W1T (n_in + 1) x 64, bias row last, then W2T 65 x
// n_out, bias row last.  Lane l holds hidden units HPL*l .. HPL*l + HPL - 1.
// Every dot product starts from the bias and accumulates in index order.
template <int G>
__device__ void policy(const BatchArgs &A, const TplDev &td, CreatureSmem &X, int slot,
                       const kr::Lanes<G> &L) {
  constexpr int H = KR_POLICY_HIDDEN;
  constexpr int HPL = H / G;  // hidden units per lane
  const int n_in = 6 * td.arms + 6, n_out = td.arms * td.segs + td.arms, lane = L.lane;
  const float *w = A.pw + (size_t)A.pw_idx[slot] * A.pw_stride;
  const float *col = w + HPL * lane;
  float hid[HPL];
  load_vec<HPL>(col + (size_t)n_in * H, hid);
#pragma unroll 4
  for (int i = 0; i < n_in; i++) {
    float wv[HPL];
    load_vec<HPL>(col + (size_t)i * H, wv);
    const float x = X.obs[i];
#pragma unroll
    for (int u = 0; u < HPL; u++) hid[u] = fmaf(wv[u], x, hid[u]);
  }
#pragma unroll
  for (int u = 0; u < HPL; u++) hid[u] = tanhf(hid[u]);
  const float *w2 = w + (size_t)H * (n_in + 1);
  for (int base = 0; base < n_out; base += G) {
    const int o = base + lane;
    const bool ok = o < n_out;
    const float *c2 = w2 + (ok ? o : 0);
    float acc = ok ? __ldg(c2 + (size_t)H * n_out) : 0.f;
#pragma unroll
    for (int j = 0; j < H; j++) {
      const float hj = __shfl_sync(L.mask, hid[j % HPL], j / HPL, G);
      if (ok) acc = fmaf(__ldg(c2 + (size_t)j * n_out), hj, acc);
    }
    if (ok) {
      const float y = tanhf(acc);
      X.ctrl[o] = o < td.arms * td.segs ? y : 0.5f * (y + 1.f);
    }
  }
  L.sync();
}

// net.js's activation: tanh, clamped to +-1 beyond +-20, stored in a Float32Array
__device__ __forceinline__ float net_act(double s) { return (float)(s > 20 ? 1.0 : (s < -20 ? -1.0 : lib_tanh(s))); }

// What the KR_CTRL_NET steps read of BatchArgs, passed by value so that the
// non-inlined calls take no address of the kernel's arguments or state.
struct NetArgs {
  NetRec *net;
  SlotMeta *meta;
  const float *pw;
  const int *pw_idx;
  int pw_stride;
  const double *rects64;
  const int *map_off;
  const double *lights;
  const int *light_off;
  const double *map_size;
  const double2 *light_tab;
  int light_T;
  double dt;
};

__device__ __forceinline__ NetArgs net_args(const BatchArgs &A) {
  return NetArgs{A.net, A.meta, A.pw, A.pw_idx, A.pw_stride, A.rects64, A.map_off, A.lights, A.light_off,
                 A.map_size, A.light_tab, A.light_T, A.dt};
}

// tickMapLights (map.js:75-83) for one light (x y r ir ph sp at lp) at sim
// time `time`: its position after the tick
__device__ __forceinline__ double2 light_tick(double2 p, const double *lp, double time, double mw, double mh,
                                              double dt) {
  const double a = time * lp[5] + lp[4];
  return make_double2(fmax(60.0, fmin(mw - 60, p.x + lib_cos(a) * 18 * dt)),
                      fmax(60.0, fmin(mh - 60, p.y + lib_sin(a * 0.8) * 18 * dt)));
}

// The light-position table (light_table_steps): block = map, thread = light;
// the sim clock summed step by step from 0 as each creature's record sums it.
__global__ void light_table_kernel(const double *lights, const int *light_off, const double *map_size, double dt,
                                   int T, double2 *tab) {
  const int map = blockIdx.x, lo = light_off[map], nl = light_off[map + 1] - lo;
  const double mw = map_size[2 * map], mh = map_size[2 * map + 1];
  for (int l = threadIdx.x; l < nl; l += blockDim.x) {
    const double *lp = lights + 6 * (size_t)(lo + l);
    double2 p = make_double2(lp[0], lp[1]);
    double time = 0.0;
    double2 *out = tab + (size_t)(lo + l) * T;
    for (int t = 0; t < T; t++) {
      time = time + dt;
      p = light_tick(p, lp, time, mw, mh, dt);
      out[t] = p;
    }
  }
}

// KR_CTRL_NET, before the step: the trainer's input vector (train.js:236-241:
// readProprio -- already in obs --, readSenses, the previous outputs),
// forwardInto (net.js:71-98; the second layer's bias is read at b2 + j, as
// the reference reads it) and decode + applyControl's tone (net.js:124-133,
// core.js:185-199).  Writes the per-motor controls and adhesion values to
// ctrl and the emission wish to the record; returns the compliance of the
// tone.  G lanes: input entries, then hidden / output units, strided.
template <int G>
__device__ __noinline__ float net_control(NetArgs N, int arms, int segs, const float *obs, float *ctrl, int slot,
                                          kr::Lanes<G> L) {
  NetRec &R = N.net[slot];
  const int lane = L.lane;
  const int np = 6 * arms + 6, ni = net_inputs(arms), no = net_outputs(arms), H = KR_NET_HIDDEN;
  constexpr int E = 2 * KR_NET_RAYS;  // echo entries, then chem 6, light 3, hearing 4, contact
  for (int q = lane; q < ni; q += G) {
    float v;
    const int r = q - np;
    if (q < np) v = obs[q];
    else if (r < E) v = (r & 1) ? R.inten[r >> 1] : R.range[r >> 1];
    else if (r < E + 6) v = 0.f;                              // chemoreception: no scent sources
    else if (r < E + 9) v = R.light_v[r - E - 6];
    else if (r < E + 13) v = 0.f;                             // hearing: no noise sources
    else if (r < E + 13 + arms) v = (float)R.contact[r - E - 13];
    else v = R.out[r - E - 13 - arms];                        // recurrent: last step's outputs
    R.x[q] = v;
  }
  L.sync();
  // device layout (net_transpose): W1T, b1, W2T, b2, W3T, b3 -- lane j of a
  // row reads word j, so a warp's loads are consecutive words.  Each lane
  // carries its units j = lane + u G as independent f64 chains; every sum
  // still runs over i in ascending order from its bias.  A product of two
  // f32 values is exact in f64, so fma(x, w, acc) rounds once exactly as
  // the reference's acc + x * w does.
  const float *w1 = N.pw + (size_t)N.pw_idx[slot] * N.pw_stride;
  const float *b1 = w1 + (size_t)ni * H, *w2 = b1 + H, *b2 = w2 + H * H, *w3 = b2 + H, *b3 = w3 + H * no;
  constexpr int U = (KR_NET_HIDDEN + G - 1) / G, UO = (KR_NET_OUT_STRIDE + G - 1) / G;
  double acc[U > UO ? U : UO];
#pragma unroll
  for (int u = 0; u < U; u++) acc[u] = lane + u * G < H ? (double)b1[lane + u * G] : 0.0;
  for (int i = 0; i < ni; i++) {
    const double xi = R.x[i];
    const float *r = w1 + i * H;
#pragma unroll
    for (int u = 0; u < U; u++)
      if (lane + u * G < H) acc[u] = fma(xi, (double)r[lane + u * G], acc[u]);
  }
#pragma unroll
  for (int u = 0; u < U; u++)
    if (lane + u * G < H) R.h[lane + u * G] = net_act(acc[u]);
  L.sync();
#pragma unroll
  for (int u = 0; u < U; u++) acc[u] = lane + u * G < H ? (double)b2[lane + u * G] : 0.0;
  for (int i = 0; i < H; i++) {
    const double hi = R.h[i];
    const float *r = w2 + i * H;
#pragma unroll
    for (int u = 0; u < U; u++)
      if (lane + u * G < H) acc[u] = fma(hi, (double)r[lane + u * G], acc[u]);
  }
#pragma unroll
  for (int u = 0; u < U; u++)
    if (lane + u * G < H) R.h[H + lane + u * G] = net_act(acc[u]);
  L.sync();
#pragma unroll
  for (int u = 0; u < UO; u++) acc[u] = lane + u * G < no ? (double)b3[lane + u * G] : 0.0;
  for (int i = 0; i < H; i++) {
    const double hi = R.h[H + i];
    const float *r = w3 + i * no;
#pragma unroll
    for (int u = 0; u < UO; u++)
      if (lane + u * G < no) acc[u] = fma(hi, (double)r[lane + u * G], acc[u]);
  }
#pragma unroll
  for (int u = 0; u < UO; u++)
    if (lane + u * G < no) R.out[lane + u * G] = net_act(acc[u]);
  L.sync();
  // decode: motor 0 of arm a takes its shoulder output, the distal motors its curl
  const int AS = arms * segs;
  for (int q = lane; q < AS; q += G) {
    const int a = q / segs;
    ctrl[q] = R.out[(q % segs) == 0 ? 1 + 3 * a : 2 + 3 * a];
  }
  for (int a = lane; a < arms; a += G) {
    const float v = R.out[3 + 3 * a];
    ctrl[AS + a] = v > 0.f ? v : 0.f;
  }
  const double tone = fmax(0.0, fmin(1.0, 0.5 + 0.5 * (double)R.out[0]));
  if (lane == 0) {
    N.meta[slot].tone_d = tone;
    R.wants_emit = (double)R.out[no - 1] > 0.3 ? 1 : 0;
  }
  L.sync();
  return (float)(1.0 / (2000.0 + tone * (400000.0 - 2000.0)));  // toneToCompliance
}

// The echo's ray march and the contact's SDF out of line: one copy each of
// the f64 rect loop (instruction-cache footprint of the per-step path).
__device__ __noinline__ double net_echo_ray(const double *rects, int n, double x, double y, double cx, double cy) {
  return echo_march(rects, n, x, y, cx, cy, kEchoRange);
}
__device__ __noinline__ double2 net_sdf(const double *rects, int n, double px, double py) {
  double d = 0.0;
  const bool ok = sdf64(rects, n, px, py, &d);
  return make_double2(ok ? 1.0 : 0.0, d);
}

// KR_CTRL_NET, after postStep: sim.time += dt, tickMapLights (map.js:75-83)
// on the creature's copy of its map's lights, then tickSenses (core.js:
// 245-267) without entities: the echo's tick (echo.js:120-127) and, when
// the net asked for it and the cooldown allows, an emission (echo.js:67-85:
// 12 rays over the fan, lanes strided, arrivals inserted in arrival order
// after equal times, as the stable sort after the push orders them); the
// light sense (light.js:90-97) and the tip contact per arm.  t: the env
// step this is the end of (the slot's step counter, from 0 at its spawn):
// below light_T the lights' positions come from the engine's table.
template <int G>
__device__ __noinline__ void net_senses(NetArgs N, int arms, const int *arm_tip, const float *px, const float *py,
                                        const float *ang, int map, int slot, int t, kr::Lanes<G> L) {
  NetRec &R = N.net[slot];
  const int lane = L.lane;
  const int ro = N.map_off[map], nR = N.map_off[map + 1] - ro;
  const double *rects = N.rects64 + 4 * (size_t)ro;
  const double x = px[0], y = py[0];
  const double heading = (double)ang[0] - kPiD * 0.5;
  const double dt = N.dt;
  const double time = R.time + dt;
  const int lo = N.light_off ? N.light_off[map] : 0, nl = N.light_off ? N.light_off[map + 1] - lo : 0;
  const double *lp = N.lights + 6 * (size_t)lo;
  // the lights move (light l on lane l), then every (sample point, light)
  // contribution on its own lane; lane 0 sums them in light order below
  if (lane < nl) {
    const int l = lane;
    double2 p;
    if (t < N.light_T) {
      p = N.light_tab[(size_t)(lo + l) * N.light_T + t];
    } else {
      p = light_tick(make_double2(R.light_xy[2 * l], R.light_xy[2 * l + 1]), lp + 6 * l, time,
                     N.map_size[2 * map], N.map_size[2 * map + 1], dt);
    }
    R.light_xy[2 * l] = p.x;
    R.light_xy[2 * l + 1] = p.y;
  }
  L.sync();
  {
    const double2 hp = lib_sincos(heading + kPiD / 2);  // light.js: receptors 26 px across the heading
    const double sp = hp.x, cp = hp.y;
    for (int q = lane; q < 3 * nl; q += G) {
      const int s = q / nl, l = q % nl;
      const double qx = s == 0 ? x + cp * 26 : (s == 1 ? x - cp * 26 : x);
      const double qy = s == 0 ? y + sp * 26 : (s == 1 ? y - sp * 26 : y);
      const double d = lib_hypot(qx - R.light_xy[2 * l], qy - R.light_xy[2 * l + 1]);
      R.lc[q] = fmax(0.0, 1 - d / lp[6 * l + 2]) * lp[6 * l + 3];
    }
  }
  L.sync();
  int emit = 0;
  if (lane == 0) {
    R.time = time;
    for (int s = 0; s < 3; s++) {  // sampleAt, light.js:99-106
      double v = 0.05;
      for (int l = 0; l < nl; l++) v += R.lc[s * nl + l];
      R.light_v[s] = (float)fmin(1.0, v);
    }
    if (R.cooldown > 0) R.cooldown -= dt;
    int k = 0;
    while (k < R.n_pending && R.p_at[k] <= time) {
      R.range[R.p_ray[k]] = R.p_range[k];
      R.inten[R.p_ray[k]] = R.p_inten[k];
      k++;
    }
    for (int q = k; q < R.n_pending; q++) {
      R.p_at[q - k] = R.p_at[q]; R.p_ray[q - k] = R.p_ray[q];
      R.p_range[q - k] = R.p_range[q]; R.p_inten[q - k] = R.p_inten[q];
    }
    R.n_pending -= k;
    if (R.wants_emit && !(R.cooldown > 0)) {
      R.cooldown = kEchoInterval;
      R.emit_count++;
      emit = 1;
    }
  }
  emit = __shfl_sync(L.mask, emit, 0, G);
  if (emit) {
    for (int i = lane; i < KR_NET_RAYS; i += G) {
      const double t = (double)i / (KR_NET_RAYS - 1);
      const double a = heading + (t - 0.5) * (kPiD * 0.85);
      const double2 ra = lib_sincos(a);
      R.ray_d[i] = net_echo_ray(rects, nR, x, y, ra.y, ra.x);
    }
    L.sync();
    if (lane == 0) {
      const double time = R.time;
      for (int i = 0; i < KR_NET_RAYS; i++) {
        const double d = R.ray_d[i];
        if (d >= kEchoRange) continue;
        const double inten = fmin(1.0, (kEchoRange * 0.22) / fmax(8.0, d * d / kEchoRange));
        const double at = time + (2 * d) / kEchoSpeed;
        if (R.n_pending >= kEchoPending) { R.dropped++; continue; }
        int q = R.n_pending;
        while (q > 0 && R.p_at[q - 1] > at) {
          R.p_at[q] = R.p_at[q - 1]; R.p_ray[q] = R.p_ray[q - 1];
          R.p_range[q] = R.p_range[q - 1]; R.p_inten[q] = R.p_inten[q - 1];
          q--;
        }
        R.p_at[q] = at; R.p_ray[q] = i;
        R.p_range[q] = (float)(d / kEchoRange); R.p_inten[q] = (float)inten;
        R.n_pending++;
      }
    }
  }
  // tip contact: near = max(0, 1 - d / 9) of the map's SDF at the tip point
  for (int a = lane; a < arms; a += G) {
    const int tip = arm_tip[a];
    const double2 t = lib_sincos((double)ang[tip]);
    const double tx = (double)px[tip] + kSegHalf * t.y, ty = (double)py[tip] + kSegHalf * t.x;
    // near is 0 unless a rect lies within 9 px: a rect whose box is 10 px
    // away or more cannot make it positive, so the SDF runs only when some
    // box is closer (the result is the same either way)
    bool close = false;
    for (int i = 0; i < nR && !close; i++) {
      const double *r = rects + 4 * i;
      const bool far = r[2] >= 0 && r[3] >= 0 &&
                       (tx <= r[0] - 10 || tx >= r[0] + r[2] + 10 || ty <= r[1] - 10 || ty >= r[1] + r[3] + 10);
      close = !far;  // NaN coordinates or extents count as close: the SDF then decides
    }
    const double2 sd = close ? net_sdf(rects, nR, tx, ty) : make_double2(0.0, 0.0);
    const double near = sd.x != 0.0 ? fmax(0.0, 1 - sd.y / 9) : 0.0;
    R.contact[a] = R.contact[a] * 0.7 + near * 0.3;
  }
  L.sync();
}

// One creature (slot) advanced by its G lanes for up to A.max_steps env steps.
// NET: the kernel instance of engines in KR_CTRL_NET mode (the other modes'
// kernels carry none of the net's code).
template <int G, bool NET, int U>
__device__ void run_creature(const BatchArgs &A, const TplDev &td, int nlv, const TplSmem &P, float *base,
                             int slot, const kr::Lanes<G> &L) {
  const int lane = L.lane;
  kr::Island S;
  CreatureSmem X;
  carve_creature(S, X, P, base, td);
  S.nlv = nlv;
  SlotMeta m = A.meta[slot];
  const int steps = min(A.max_steps, m.horizon - m.step);
  if (steps <= 0) return;
  const int arms = td.arms, AS = td.arms * td.segs;
  float4 *gst = A.grip + (size_t)slot * KR_BATCH_MAX_ARMS;
  float2 *glam = A.glam + (size_t)slot * KR_BATCH_MAX_ARMS;
  double2 *cdp = A.cd + (size_t)slot * KR_BATCH_MAX_ARMS;
  // the committed state into shared memory (the slot's block is SoA, kBodyPad per field)
  float *hbm = A.state + (size_t)slot * kStateStride;
  for (int i = lane; i < td.nb; i += G) {
    S.px[i] = hbm[i]; S.py[i] = hbm[kBodyPad + i]; S.vx[i] = hbm[2 * kBodyPad + i];
    S.vy[i] = hbm[3 * kBodyPad + i]; S.ang[i] = hbm[4 * kBodyPad + i]; S.av[i] = hbm[5 * kBodyPad + i];
  }
  for (int k = lane; k < td.nc; k += G) { S.lamX[k] = 0.f; S.lamY[k] = 0.f; }
  S.comp_m = m.comp;
  double cd = 0.0;  // reflex cooldown of arm `lane` (its f64 break force stays in cdp)
  L.sync();
  if (lane < arms) {
    reinterpret_cast<float4 *>(S.anc)[lane] = gst[lane];
    const float2 gl = glam[lane];
    const int k = P.arm_grip[lane];
    S.lamX[k] = gl.x; S.lamY[k] = gl.y;
    cd = cdp[lane].x;
  }
  const float *cin = A.ctrl_cur + (size_t)slot * kCtrlStride;
  for (int q = lane; q < AS + arms; q += G) X.ctrl[q] = cin[q];
  L.sync();
  const float4 *rects = A.rects + A.map_off[m.map];
  const int nR = A.map_off[m.map + 1] - A.map_off[m.map];
  const float cull_d = fmaxf(A.map_cull[m.map], td.r_max + 2.f + kr::kCullSlack + 1.f);
  int halt_next = 0;  // the stop word as loaded during the previous step
  for (int s = 0; s < steps; s++) {
    if (A.stop) {
      if (s > 0 && __shfl_sync(L.mask, halt_next, L.base)) break;
      if (lane == 0) halt_next = *reinterpret_cast<const volatile int *>(A.stop);
    }
    const int t = m.step;
    // 1. proprioception of the current state
    if (A.obs_ring > 0 || m.ctrl == KR_CTRL_POLICY || (NET && m.ctrl == KR_CTRL_NET)) {
      const unsigned att = proprio<G>(A, td, P, S, X, m, cdp, L);
      if (A.obs_ring > 0) {
        float *o = A.obs + ((size_t)slot * A.obs_ring + (t % A.obs_ring)) * KR_OBS_STRIDE;
        for (int q = lane; q < 6 * arms + 6; q += G) o[q] = X.obs[q];
        if (lane == 0) o[KR_OBS_STRIDE - 1] = __uint_as_float(att);
      }
    }
    // 2. controls
    if (m.ctrl == KR_CTRL_STREAM) {
      if (t % A.ctrl_period == 0) {
        // the redraw's arms x (segs + 1) draws, in the stream's order (per
        // arm its motors, then its adhesion), split over the lanes
        const int per = td.segs + 1, nd = arms * per;
        for (int d = lane; d < nd; d += G) {
          const double r = mulberry_at(m.rng + (uint32_t)(d + 1) * kMulberryStep);
          const int a = d / per, j = d - a * per;
          if (j < td.segs) X.ctrl[a * td.segs + j] = (float)(r * 2 - 1);
          else X.ctrl[AS + a] = (float)r;
        }
        m.rng += (uint32_t)nd * kMulberryStep;
      }
    } else if (m.ctrl == KR_CTRL_POLICY) {
      policy<G>(A, td, X, slot, L);
    } else if constexpr (NET) {
      if (m.ctrl == KR_CTRL_NET) S.comp_m = net_control<G>(net_args(A), arms, td.segs, X.obs, X.ctrl, slot, L);
    }
    L.sync();
    // 3. applyControl: targets (clamped) and the reflex, core.js:183-220
    for (int mo = lane; mo < AS; mo += G) {
      const double lim = (mo % td.segs) == 0 ? kPiD * 0.62 : kPiD * 0.42;
      S.tgt_m[mo] = (float)fmax(-lim, fmin(lim, (double)X.ctrl[mo]));
    }
    if (lane < arms) {
      const int a = lane, k = P.arm_grip[a], tip = P.arm_tip[a];
      float *an = S.anc + 4 * a;
      const double adh = fmax(0.0, fmin(1.0, (double)X.ctrl[AS + a]));
      double c = cd;
      if (c > 0) c -= A.dt;
      if (an[3] != 0.f) {
        if (adh > 0.08 && c <= 0) {
          const double slip = lib_hypot((double)S.vx[tip], (double)S.vy[tip]);
          if (slip < A.slip_max) {
            const double ta = (double)S.ang[tip];
            an[0] = (float)((double)S.px[tip] + kSegHalf * lib_cos(ta));
            an[1] = (float)((double)S.py[tip] + kSegHalf * lib_sin(ta));
            const double brk = 40.0 + 860.0 * adh;
            cdp[a].y = brk;
            an[2] = (float)brk;
            an[3] = 0.f;
            S.lamX[k] = 0.f; S.lamY[k] = 0.f;
          } else {
            c = A.cooldown;
          }
        }
      } else {
        const double brk = 40.0 + 860.0 * adh;
        cdp[a].y = brk;
        an[2] = (float)brk;
        if (adh < 0.04) an[3] = 1.f;
      }
      cd = c;
    }
    L.sync();
    // 4. the XPBD step
    kr::island_step<kr::CompactAccess, G, U>(A.K, S, rects, nR, cull_d, L, td.off_max + 1.f);
    // 5. postStep, core.js:297-356 (f64 on the f32 state, as the
    //    reference's hybrid loop runs it on the mirrored state)
    //    The accumulators are read and written through the slot's HBM
    //    record by lane 0 (they do not live in every lane's registers).
    //    The two distances (the step's and the spawn point's) come from one
    //    call on two lanes, beside lane 0's sincos of the heading.
    {
      const SlotMeta &gr = A.meta[slot];
      const double x = S.px[0], y = S.py[0];
      const double hx = lane == 1 ? x - gr.spawn_x : x - gr.last_x;
      const double hy = lane == 1 ? y - gr.spawn_y : y - gr.last_y;
      const double hv = lib_hypot(hx, hy);
      const double d_spawn_l = __shfl_sync(L.mask, hv, L.base + 1);
      if (lane == 0) {
        SlotMeta &g = A.meta[slot];
        const double angle = S.ang[0], av = S.av[0];
        const double dx = hx, dy = hy;
        const double step_dist = hv;
        g.path_len += step_dist;
        g.angular_accum += fabs(av) * A.h64 * A.substeps;
        const double fa = angle - kPiD * 0.5;
        const double2 fsc = lib_sincos(fa);
        const double sf = fsc.x, cf = fsc.y;
        const double fwd = dx * cf + dy * sf;
        if (fwd > 0) g.forward_prog += fwd;
        int anchored = 0;
        unsigned now = 0;
        for (int a = 0; a < arms; a++)
          if (S.anc[4 * a + 3] == 0.f) { anchored++; now |= 1u << a; }
        const double d_spawn = d_spawn_l;
        if (anchored > 0) {
          g.anchored_steps++;
          if (d_spawn > g.spawn_dist_max) { g.grip_pull_prog += d_spawn - g.spawn_dist_max; g.spawn_dist_max = d_spawn; }
        }
        if (anchored == 0 && step_dist > 0.3) g.free_move += step_dist;
        g.energy += (g.tone_d * 0.0006 + step_dist * 0.0004) * arms;
        const unsigned was = g.arm_anchored;
        if (anchored > 0 && !(was & 0x100u)) g.grip_cycles++;
        const int newly = __popc(now & ~was & 0xffu);
        g.attach_events += newly;
        if (newly > 0 && anchored - newly > 0) g.strides += newly;
        g.arm_anchored = now | (anchored > 0 ? 0x100u : 0u);
        g.max_disp = fmax(g.max_disp, d_spawn);
        g.last_x = x; g.last_y = y;
      }
    }
    if constexpr (NET) {
      if (m.ctrl == KR_CTRL_NET) net_senses<G>(net_args(A), arms, P.arm_tip, S.px, S.py, S.ang, m.map, slot, t, L);
    }
    m.step = t + 1;
  }
  // write back: the committed state, grips, cooldowns, controls, the meta fields kept in registers
  L.sync();
  for (int i = lane; i < td.nb; i += G) {
    hbm[i] = S.px[i]; hbm[kBodyPad + i] = S.py[i]; hbm[2 * kBodyPad + i] = S.vx[i];
    hbm[3 * kBodyPad + i] = S.vy[i]; hbm[4 * kBodyPad + i] = S.ang[i]; hbm[5 * kBodyPad + i] = S.av[i];
  }
  if (lane < arms) {
    const int k = P.arm_grip[lane];
    gst[lane] = reinterpret_cast<const float4 *>(S.anc)[lane];
    glam[lane] = make_float2(S.lamX[k], S.lamY[k]);
    cdp[lane].x = cd;
  }
  float *cout = A.ctrl_cur + (size_t)slot * kCtrlStride;
  for (int q = lane; q < AS + arms; q += G) cout[q] = X.ctrl[q];
  if (lane == 0) {  // the fields this loop keeps in registers; postStep's are in place
    SlotMeta &g = A.meta[slot];
    g.step = m.step;
    g.rng = m.rng;
    g.prev_vx = m.prev_vx;
    g.prev_vy = m.prev_vy;
    // the record is final once the count includes this creature: the server
    // copies a request's records back (copy engine) while the launch still runs
    if (A.tag_done && m.step >= m.horizon) {
      __threadfence_system();
      atomicAdd(A.tag_done + m.pad, 1);
    }
  }
}

template <int G, bool NET, int U>
__global__ void __launch_bounds__(32 * kMaxW, 1) batch_kernel(BatchArgs A) {
  constexpr int CPW = 32 / G;  // creatures per warp
  constexpr int V = G == 32 ? 0 : G == 16 ? 1 : 2;  // kr::schedule_index(G): the schedule for G lanes
  extern __shared__ __align__(16) float smem[];
  __shared__ int s_group;
  const int warp = threadIdx.x >> 5, wl = threadIdx.x & 31;
  const kr::Lanes<G> L(wl);
  const int c = warp * CPW + wl / G;  // creature entry of this lane group
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0)
      s_group = A.stop && *reinterpret_cast<const volatile int *>(A.stop) ? A.n_groups : atomicAdd(A.queue, 1);
    __syncthreads();
    const int g = s_group;
    if (g >= A.n_groups) return;
    const int first = A.groups[g * A.cpc];
    const TplDev td = A.tpl[A.meta[first].tpl];
    TplSmem P;
    carve_tpl(P, smem, td);
    // stage the template statics (whole CTA)
    for (int i = threadIdx.x; i < td.nb; i += blockDim.x) {
      P.im[i] = A.T.im[td.o_b + i]; P.ii[i] = A.T.ii[td.o_b + i]; P.zero[i] = 0.f;
      P.boff[i] = A.T.boff[td.o_b + i]; P.bcnt[i] = A.T.bcnt[td.o_b + i];
    }
    for (int k = threadIdx.x; k < td.nc; k += blockDim.x) {
      const int o = td.o_c[V] + k;
      P.ab[k] = A.T.ab[o]; P.type[k] = A.T.type[o]; P.motor[k] = A.T.motor[o]; P.garm[k] = A.T.garm[o];
      P.lax[k] = A.T.lax[o]; P.lay[k] = A.T.lay[o]; P.lbx[k] = A.T.lbx[o]; P.lby[k] = A.T.lby[o];
      P.rest[k] = A.T.rest[o]; P.minA[k] = A.T.minA[o]; P.maxA[k] = A.T.maxA[o];
    }
    for (int l = threadIdx.x; l <= td.nlv[V]; l += blockDim.x) P.lvl[l] = A.T.lvl[td.o_l[V] + l];
    for (int p = threadIdx.x; p < td.np; p += blockDim.x) {
      P.plx[p] = A.T.plx[td.o_p + p]; P.ply[p] = A.T.ply[td.o_p + p]; P.pr[p] = A.T.pr[td.o_p + p];
      P.pbody[p] = A.T.pbody[td.o_p + p];
    }
    for (int a = threadIdx.x; a < td.arms; a += blockDim.x) {
      P.arm_tip[a] = A.T.arm_tip[td.o_a + a]; P.arm_grip[a] = A.T.arm_grip[td.o_g[V] + a];
      P.arm_seg0[a] = A.T.arm_seg0[td.o_a + a];
    }
    for (int q = threadIdx.x; q < td.arms * td.segs; q += blockDim.x) P.arm_segs[q] = A.T.arm_segs[td.o_s + q];
    __syncthreads();
    const int slot = c < A.cpc ? A.groups[g * A.cpc + c] : -1;
    if (slot >= 0) {
      float *base = smem + tpl_smem_words(td.nb, td.nc, td.np) +
                    c * creature_smem_words(td.nb, td.nc, td.np, td.arms, td.segs);
      run_creature<G, NET, U>(A, td, td.nlv[V], P, base, slot, L);
    }
  }
}

// one block per spawned creature: copies its pose and metadata into the slot,
// clears its grips and controls, and measures its spawn reach (16 threads,
// one ray each; init's spawn_reach holds the body's arm reach on entry);
// with net records, clears the slot's record and places its copy of the
// map's lights
__global__ void spawn_kernel(float *state, float4 *grip, float2 *glam, double2 *cd, SlotMeta *meta,
                             float *ctrl, const int *slots, const float *pose, const SlotMeta *init, int n,
                             const double *rects, const int *map_off, RayDirs rays, NetRec *net,
                             const double *lights, const int *light_off) {
  __shared__ double ray_d[16];
  const int i = blockIdx.x;
  if (i >= n) return;
  if (net) {
    NetRec *R = net + slots[i];
    uint32_t *words = reinterpret_cast<uint32_t *>(R);
    for (int q = threadIdx.x; q < (int)(sizeof(NetRec) / 4); q += blockDim.x) words[q] = 0u;
    __syncthreads();
    if (light_off && threadIdx.x < 2 * KR_NET_MAX_LIGHTS) {
      const int map = init[i].map, lo = light_off[map], nl = light_off[map + 1] - lo, l = threadIdx.x >> 1;
      if (l < nl) R->light_xy[threadIdx.x] = lights[6 * (size_t)(lo + l) + (threadIdx.x & 1)];
    }
  }
  if (threadIdx.x < 16) {
    const SlotMeta &m = init[i];
    const int o = map_off[m.map], nr = map_off[m.map + 1] - o;
    ray_d[threadIdx.x] = reach_ray(rects + 4 * (size_t)o, nr, m.spawn_reach, m.spawn_x, m.spawn_y,
                                   rays.c[threadIdx.x], rays.s[threadIdx.x]);
  }
  __syncthreads();
  const int slot = slots[i];
  const float *src = pose + (size_t)i * kStateStride;
  float *dst = state + (size_t)slot * kStateStride;
  for (int q = threadIdx.x; q < kStateStride; q += blockDim.x) dst[q] = src[q];
  if (threadIdx.x < KR_BATCH_MAX_ARMS) {
    grip[(size_t)slot * KR_BATCH_MAX_ARMS + threadIdx.x] = make_float4(0.f, 0.f, 0.f, 1.f);
    glam[(size_t)slot * KR_BATCH_MAX_ARMS + threadIdx.x] = make_float2(0.f, 0.f);
    cd[(size_t)slot * KR_BATCH_MAX_ARMS + threadIdx.x] = make_double2(0.0, 0.0);
  }
  for (int q = threadIdx.x; q < kCtrlStride; q += blockDim.x) ctrl[(size_t)slot * kCtrlStride + q] = 0.f;
  if (threadIdx.x == 0) {
    SlotMeta m = init[i];
    double sum = 0, best = 0;
    for (int k = 0; k < 16; k++) {
      sum += ray_d[k];
      if (ray_d[k] > best) best = ray_d[k];
    }
    const double v = (sum / 16) * 0.55 + best * 0.45;
    m.spawn_reach = 70.0 < v ? v : 70.0;
    meta[slot] = m;
  }
}

// every slot's step counter into one contiguous array (read back after a
// time slice: a preempted slice leaves each creature at its own step)
__global__ void step_counts_kernel(const SlotMeta *meta, int n, int *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = meta[i].step;
}

}  // namespace


namespace {
thread_local std::string g_batch_error;

template <typename T>
cudaError_t upload_vec(T **d, const std::vector<T> &v) {
  if (*d) cudaFree(*d);
  *d = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(d), std::max<size_t>(v.size(), 1) * sizeof(T));
  if (e != cudaSuccess || v.empty()) return e;
  return cudaMemcpy(*d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// relative cost of one env step of a template (constraint and collision work)
double tpl_cost(const TplDev &d) { return (double)d.nc + 0.5 * (double)d.np; }
}  // namespace

namespace krb {

cudaStream_t part_stream(const kr_batch *b, const Part &p) { return p.stream ? p.stream : b->stream; }

// score, src/sim/fitness.js:115-172 without prey (preyHit = preyNear = 0),
// maxAngSpeed 18 and dt 1/60 as the trainer calls it: the terms in
// TERM_ORDER, summed in f64 in that order
static double fitness_score(const SlotMeta &c) {
  const double steps = std::max(1, c.step), path = c.path_len, disp = c.max_disp;
  const double reach = c.spawn_reach > 0 ? c.spawn_reach : 300;
  const double reach_frac = std::min(1.2, disp / reach);
  const double directed = path > 1 ? std::min(1.0, disp / path) : 0;
  const double spin_budget = steps * 18 * (1.0 / 60);
  const double heading_hold = 1 - std::min(1.0, c.angular_accum / std::max(1e-6, spin_budget));
  const double mean_speed = path / steps / 60;
  const double efficiency = c.forward_prog / std::max(0.5, c.energy > 0 ? c.energy : 0.5);
  const double progress_base = c.grip_pull_prog * 2.6 + reach_frac * 320;
  const double stride_frac = std::min((double)c.strides, 60.0) / 60.0;
  const double prog_gate = std::min(1.0, disp / std::max(1e-6, 0.25 * reach));
  const double t[12] = {c.grip_pull_prog * 2.6,
                        progress_base * 0.5 * stride_frac,
                        reach_frac * 320,
                        directed * 70 * prog_gate,
                        heading_hold * 28 * prog_gate,
                        std::min(1.0, mean_speed) * 14 * prog_gate,
                        std::min(20.0, efficiency) * 3 * prog_gate,
                        -(c.angular_accum * 0.55 * 0.02),
                        -(c.free_move * 0.05),
                        -(c.energy * 0.30),
                        0.0,
                        0.0};
  double s = 0;
  for (double v : t) s += v;
  return std::isfinite(s) ? s : 0;
}

void slot_metrics(const SlotMeta &m, double *o) {
  o[0] = fitness_score(m); o[1] = m.step; o[2] = m.path_len; o[3] = m.max_disp; o[4] = m.spawn_reach;
  o[5] = m.angular_accum; o[6] = m.forward_prog; o[7] = m.grip_pull_prog; o[8] = m.anchored_steps;
  o[9] = m.free_move; o[10] = m.energy; o[11] = m.grip_cycles; o[12] = m.strides; o[13] = m.attach_events;
  o[14] = m.last_x; o[15] = m.last_y;
}

void free_part(Part &p) {
  if (p.d_groups) cudaFree(p.d_groups);
  if (p.h_groups) cudaFreeHost(p.h_groups);
  if (p.d_queue) cudaFree(p.d_queue);
  if (p.staged) cudaEventDestroy(p.staged);
  if (p.ev0) cudaEventDestroy(p.ev0);
  if (p.ev1) cudaEventDestroy(p.ev1);
  p = Part{};
}

void transpose_policy(const float *pub, int arms, int segs, float *dev) {
  const int n = policy_param_count(arms, segs);
  for (int p = 0; p < n; p++) dev[policy_device_index(arms, segs, p)] = pub[p];
}

int ensure_template(kr_batch *b, int arms, int segs) {
  auto key = std::make_pair(arms, segs);
  auto it = b->tpl_index.find(key);
  if (it != b->tpl_index.end()) return it->second;
  kr::Template t;
  std::string err;
  if (!kr::build_template(arms, segs, &t, &err)) return -1;
  const int id = (int)b->tpls.size();
  b->tpls.push_back(std::move(t));
  b->tpl_index[key] = id;
  return id;
}

int upload_templates(kr_batch *b) {
  std::vector<float> im, ii, lax, lay, lbx, lby, rest, minA, maxA, plx, ply, pr;
  std::vector<int> boff, bcnt, ab, type, motor, garm, lvl, pbody, tip, grip, seg0, segs;
  b->h_tpl.clear();
  for (const auto &t : b->tpls) {
    TplDev d{};
    d.nb = t.nb; d.nc = t.nc; d.np = t.np; d.arms = t.arms; d.segs = t.segs;
    d.r_max = t.r_max; d.off_max = t.off_max; d.reach = t.reach;
    d.o_b = (int)im.size(); d.o_p = (int)plx.size(); d.o_a = (int)tip.size(); d.o_s = (int)segs.size();
    im.insert(im.end(), t.im.begin(), t.im.end()); ii.insert(ii.end(), t.ii.begin(), t.ii.end());
    boff.insert(boff.end(), t.boff.begin(), t.boff.end()); bcnt.insert(bcnt.end(), t.bcnt.begin(), t.bcnt.end());
    for (int v = 0; v < kr::kSchedules; v++) {
      const kr::Schedule &S = t.sched[v];
      d.nlv[v] = S.nlv;
      d.o_c[v] = (int)ab.size(); d.o_l[v] = (int)lvl.size(); d.o_g[v] = (int)grip.size();
      ab.insert(ab.end(), S.ab.begin(), S.ab.end()); type.insert(type.end(), S.type.begin(), S.type.end());
      motor.insert(motor.end(), S.motor.begin(), S.motor.end());
      std::vector<int> ga(t.nc, -1);
      for (int a = 0; a < t.arms; a++) ga[S.arm_grip[a]] = a;
      garm.insert(garm.end(), ga.begin(), ga.end());
      lax.insert(lax.end(), S.lax.begin(), S.lax.end()); lay.insert(lay.end(), S.lay.begin(), S.lay.end());
      lbx.insert(lbx.end(), S.lbx.begin(), S.lbx.end()); lby.insert(lby.end(), S.lby.begin(), S.lby.end());
      rest.insert(rest.end(), S.rest.begin(), S.rest.end());
      minA.insert(minA.end(), S.minA.begin(), S.minA.end()); maxA.insert(maxA.end(), S.maxA.begin(), S.maxA.end());
      lvl.insert(lvl.end(), S.lvl.begin(), S.lvl.end());
      grip.insert(grip.end(), S.arm_grip.begin(), S.arm_grip.end());
    }
    plx.insert(plx.end(), t.plx.begin(), t.plx.end()); ply.insert(ply.end(), t.ply.begin(), t.ply.end());
    pr.insert(pr.end(), t.pr.begin(), t.pr.end()); pbody.insert(pbody.end(), t.pbody.begin(), t.pbody.end());
    tip.insert(tip.end(), t.arm_tip.begin(), t.arm_tip.end());
    seg0.insert(seg0.end(), t.arm_seg0.begin(), t.arm_seg0.end());
    segs.insert(segs.end(), t.arm_segs.begin(), t.arm_segs.end());
    b->h_tpl.push_back(d);
  }
  // the device may still read the old tables in a queued launch
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return b->cuda_fail(e, "upload(templates) sync");
  void **A = b->d_tpl_arrays;
#define UP(i, vec) if (e == cudaSuccess) e = upload_vec(reinterpret_cast<decltype(vec.data()) *>(&A[i]), vec)
  UP(0, im); UP(1, ii); UP(2, boff); UP(3, bcnt); UP(4, ab); UP(5, type); UP(6, motor); UP(7, lax);
  UP(8, lay); UP(9, lbx); UP(10, lby); UP(11, rest); UP(12, minA); UP(13, maxA); UP(14, lvl);
  UP(15, plx); UP(16, ply); UP(17, pr); UP(18, pbody); UP(19, tip); UP(20, grip); UP(21, seg0);
  UP(22, garm);
#undef UP
  if (e != cudaSuccess) return b->cuda_fail(e, "upload(templates)");
  int *d_segs = nullptr;
  e = upload_vec(&d_segs, segs);
  if (e != cudaSuccess) return b->cuda_fail(e, "upload(template segments)");
  TplArrays &T = b->T;
  T.im = (const float *)A[0]; T.ii = (const float *)A[1]; T.boff = (const int *)A[2]; T.bcnt = (const int *)A[3];
  T.ab = (const int *)A[4]; T.type = (const int *)A[5]; T.motor = (const int *)A[6];
  T.lax = (const float *)A[7]; T.lay = (const float *)A[8]; T.lbx = (const float *)A[9]; T.lby = (const float *)A[10];
  T.rest = (const float *)A[11]; T.minA = (const float *)A[12]; T.maxA = (const float *)A[13];
  T.lvl = (const int *)A[14]; T.plx = (const float *)A[15]; T.ply = (const float *)A[16]; T.pr = (const float *)A[17];
  T.pbody = (const int *)A[18]; T.arm_tip = (const int *)A[19]; T.arm_grip = (const int *)A[20];
  T.arm_seg0 = (const int *)A[21]; T.garm = (const int *)A[22];
  if (T.arm_segs) cudaFree(const_cast<int *>(T.arm_segs));
  T.arm_segs = d_segs;
  if ((e = upload_vec(&b->d_tpl, b->h_tpl)) != cudaSuccess) return b->cuda_fail(e, "upload(template table)");
  b->shape_dirty = true;
  return KR_OK;
}

// Launch shape: creatures per group of every template and the dynamic shared
// memory of a CTA.  A CTA gets an equal share of the SM's shared memory for
// ctas_per_sm CTAs (default: 16 warps per SM); a template's group holds as
// many creatures as fit in that share, at most W * 32 / G.
int plan_shape(kr_batch *b) {
  b->cpc = b->W * (32 / b->G);
  const int ctas = b->ctas_per_sm > 0 ? b->ctas_per_sm : std::max(1, 16 / b->W);
  long budget = std::min<long>(b->smem_optin, (long)b->smem_per_sm / ctas - b->smem_reserved) - 64;
  budget = (budget / 16) * 16;
  const long words = budget / 4;
  b->tpl_cpg.assign(b->h_tpl.size(), 0);
  size_t need_max = 16;
  for (size_t t = 0; t < b->h_tpl.size(); t++) {
    const TplDev &d = b->h_tpl[t];
    const long tw = tpl_smem_words(d.nb, d.nc, d.np);
    const long cw = creature_smem_words(d.nb, d.nc, d.np, d.arms, d.segs);
    const long fit = (words - tw) / cw;
    if (fit < 1)
      return b->fail(KR_ERR_CAPACITY, "body " + std::to_string(d.arms) + "x" + std::to_string(d.segs) +
                                          " does not fit the shared memory of " + std::to_string(ctas) +
                                          " CTAs per SM");
    const int cpg = (int)std::min<long>(b->cpc, fit);
    b->tpl_cpg[t] = cpg;
    need_max = std::max(need_max, (size_t)(tw + (long)cpg * cw) * sizeof(float));
  }
  b->smem_dyn = need_max;
  b->shape_dirty = false;
  b->main.dirty = true;
  return KR_OK;
}

// Groups of up to tpl_cpg slots of one template.  Creatures of one template
// are sorted by remaining steps, so the creatures that share a warp finish
// together; groups are queued by their work (steps this launch x template
// cost), largest first, so the launch ends on short groups.
void gather_live(kr_batch *b, Part &p) {
  p.g_live.clear();
  p.g_tpl.clear();
  p.g_rem.clear();
  p.g_ctrl.clear();
  p.g_per_arm = 0;
  p.g_net = 0;
  auto take = [&](int s) {
    const int r = b->h_remaining[s];
    if (r <= 0) return;
    const SlotMeta &m = b->h_meta[s];
    if (m.horizon <= 0) return;
    p.g_live.push_back(s);
    p.g_tpl.push_back(m.tpl);
    p.g_rem.push_back(r);
    p.g_ctrl.push_back(m.ctrl);
    p.g_per_arm += m.ctrl == KR_CTRL_POLICY || m.ctrl == KR_CTRL_NET;
    p.g_net += m.ctrl == KR_CTRL_NET;
  };
  if (p.all) {
    for (int s = 0; s < b->capacity; s++) take(s);
  } else {
    for (int s : p.slots) take(s);
  }
  p.gathered = true;
}

int build_groups(kr_batch *b, Part &p, int max_steps) {
  // the live slots, gathered once (by launch_part's shape choice just
  // before, or here); a gather is used by one build only
  const bool fresh = p.gathered;
  p.gathered = false;
  if (b->shape_dirty) {
    int rc = plan_shape(b);
    if (rc != KR_OK) return rc;
  }
  if (!fresh) gather_live(b, p);
  p.gathered = false;
  const int n_live = (int)p.g_live.size();
  for (int i = 0; i < n_live; i++) {
    const int ctrl = p.g_ctrl[i];
    if (ctrl != KR_CTRL_NET && ctrl != KR_CTRL_POLICY) continue;
    const int s = p.g_live[i];
    if (ctrl == KR_CTRL_NET) {
      if (!b->d_pw || b->h_pw_idx.size() != (size_t)b->capacity)
        return b->fail(KR_ERR_STATE, "slot " + std::to_string(s) + ": net control without kr_batch_set_net");
      if (b->h_pw_arms[b->h_pw_idx[s]] != b->tpls[p.g_tpl[i]].arms)
        return b->fail(KR_ERR_STATE, "slot " + std::to_string(s) + ": its genome was set for another arm "
                                         "count (kr_batch_set_net after the spawn)");
      continue;
    }
    if (!b->d_pw || b->h_pw_idx.size() != (size_t)b->capacity)
      return b->fail(KR_ERR_STATE, "slot " + std::to_string(s) + ": policy control without kr_batch_set_policy");
    if (b->h_pw_tpl[b->h_pw_idx[s]] != p.g_tpl[i])
      return b->fail(KR_ERR_STATE, "slot " + std::to_string(s) + ": its individual's weights were laid out for "
                                       "another body shape (kr_batch_set_policy after the spawn)");
  }
  // by template, then longest remaining first, ties in slot-list order
  lpt_order(n_live, p.g_tpl.data(), p.g_rem.data(), p.perm, p.keys, p.keys2, p.perm2);
  std::vector<int> &live = p.s_live;
  live.resize(n_live);
  for (int i = 0; i < n_live; i++) live[i] = p.g_live[p.perm[i]];
  // Group size per template.  When the live creatures fill less than one
  // wave of the resident CTAs, smaller groups (whole warps) spread them over
  // every SM instead of packing a few SMs.
  const int cpw = 32 / b->G;
  const int ctas = b->ctas_per_sm > 0 ? b->ctas_per_sm : std::max(1, 16 / b->W);
  const long slots = (long)b->n_sm * ctas;
  std::vector<int> n_t(b->h_tpl.size(), 0), size_t_(b->h_tpl.size(), 0);
  for (int i = 0; i < n_live; i++) n_t[p.g_tpl[i]]++;
  long full_groups = 0;
  for (size_t t = 0; t < n_t.size(); t++)
    if (n_t[t]) full_groups += (n_t[t] + b->tpl_cpg[t] - 1) / b->tpl_cpg[t];
  for (size_t t = 0; t < n_t.size(); t++) {
    size_t_[t] = b->tpl_cpg[t];
    if (!n_t[t] || full_groups >= slots || n_live == 0) continue;
    const long want = std::max<long>(1, (long)((double)slots * n_t[t] / (double)n_live));
    int sz = (int)((n_t[t] + want - 1) / want);
    sz = ((sz + cpw - 1) / cpw) * cpw;
    size_t_[t] = std::max(cpw, std::min(b->tpl_cpg[t], sz));
  }
  std::vector<std::pair<double, int>> order;  // (work, first index into live)
  std::vector<int> starts, sizes;
  for (int i = 0; i < n_live;) {
    const int t = p.g_tpl[p.perm[i]];
    const int st = i;
    int n = 0;
    while (i < n_live && n < size_t_[t] && p.g_tpl[p.perm[i]] == t) { i++; n++; }
    const double work = (double)std::min(max_steps, p.g_rem[p.perm[st]]) * tpl_cost(b->h_tpl[t]);
    order.push_back({work, (int)starts.size()});
    starts.push_back(st);
    sizes.push_back(n);
  }
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<double, int> &x, const std::pair<double, int> &y) { return x.first > y.first; });
  const size_t need = std::max<size_t>(order.size() * b->cpc, 1);
  cudaStream_t st = part_stream(b, p);
  if (p.staged_pending) {
    cudaError_t e = cudaEventSynchronize(p.staged);
    if (e != cudaSuccess) return b->cuda_fail(e, "groups staging sync");
    p.staged_pending = false;
  }
  if (!p.h_groups || p.ch_groups < need) {
    if (p.h_groups) cudaFreeHost(p.h_groups);
    p.h_groups = nullptr;
    cudaError_t e = cudaMallocHost(&p.h_groups, need * sizeof(int));
    if (e != cudaSuccess) return b->cuda_fail(e, "cudaMallocHost(groups)");
    p.ch_groups = need;
  }
  if (!p.d_groups || p.c_groups < need) {
    if (p.d_groups) {
      cudaStreamSynchronize(st);
      cudaFree(p.d_groups);
    }
    p.d_groups = nullptr;
    cudaError_t e = cudaMalloc(&p.d_groups, need * sizeof(int));
    if (e != cudaSuccess) return b->cuda_fail(e, "cudaMalloc(groups)");
    p.c_groups = need;
  }
  if (!p.d_queue) {
    cudaError_t e = cudaMalloc(&p.d_queue, sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.staged, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&p.ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&p.ev1);
    if (e != cudaSuccess) return b->cuda_fail(e, "part setup");
  }
  std::fill(p.h_groups, p.h_groups + order.size() * b->cpc, -1);
  for (size_t g = 0; g < order.size(); g++) {
    const int k = order[g].second;
    for (int q = 0; q < sizes[k]; q++) p.h_groups[g * b->cpc + q] = live[starts[k] + q];
  }
  if (!order.empty()) {
    cudaError_t e = cudaMemcpyAsync(p.d_groups, p.h_groups, order.size() * b->cpc * sizeof(int),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(p.staged, st);
    if (e != cudaSuccess) return b->cuda_fail(e, "upload(groups)");
    p.staged_pending = true;
    p.h2d_bytes += order.size() * b->cpc * sizeof(int);
  }
  p.n_groups = (int)order.size();
  p.dirty = false;
  return KR_OK;
}

}  // namespace krb

namespace {
template <int G>
cudaError_t launch_g(const BatchArgs &A, kr_batch *b, cudaStream_t st, int n_groups, int *grid_out) {
  auto *fn = b->unroll == 2 ? (b->d_net ? batch_kernel<G, true, 2> : batch_kernel<G, false, 2>)
                            : (b->d_net ? batch_kernel<G, true, 1> : batch_kernel<G, false, 1>);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->smem_dyn);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * b->W, b->smem_dyn);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) { *grid_out = 0; return cudaSuccess; }
  if (b->ctas_per_sm > 0) per_sm = std::min(per_sm, b->ctas_per_sm);
  const int grid = std::max(1, std::min(n_groups, per_sm * b->n_sm));
  *grid_out = grid;
  fn<<<grid, 32 * b->W, b->smem_dyn, st>>>(A);
  return cudaGetLastError();
}
}  // namespace

namespace krb {

// Few creatures (under 16 per SM): one per warp, the shortest step latency;
// up to 96 per SM two per warp; beyond, four per warp, the most
// creature-steps per issue slot (measured on the 16k workload).
// Proprioception and the fused policy run per arm, so creatures that need
// them pack four per warp from 16 per SM on.
int auto_lanes(const kr_batch *b, long live, long per_arm) {
  const bool arm_heavy = b->d.obs_ring > 0 || 2 * per_arm > live;
  return live < 16L * b->n_sm ? 32 : (arm_heavy || live >= 96L * b->n_sm) ? 8 : 16;
}

int launch_part(kr_batch *b, Part &p, int max_steps, bool timed) {
  if (b->tpls.empty()) return KR_OK;
  if (b->d.control_mode == KR_CTRL_POLICY && !b->d_pw)
    return b->fail(KR_ERR_STATE, "policy control without kr_batch_set_policy");
  if (b->auto_shape && p.dirty) {
    gather_live(b, p);  // build_groups below takes the same gather
    const int g = auto_lanes(b, (long)p.g_live.size(), p.g_per_arm);
    // at 8 lanes, creatures under the reference net or keeping an
    // observation ring run faster as one CTA of 16 warps per SM than as two
    // of 8 (served net ES stream 2.60e7 -> 2.90e7 creature-steps/s; 65k
    // creatures with 128-step rings 4.32e7 -> 4.54e7); under the fused
    // policy the two are within noise, and stream controls keep 8
    const bool wide = b->d.obs_ring > 0 || 2 * p.g_net > (long)p.g_live.size();
    const int w = g == 32 ? 4 : (g == 8 && wide) ? 16 : 8;
    if (g != b->G || w != b->W) {
      b->G = g;
      b->W = w;
      b->shape_dirty = true;
    }
  }
  if (p.dirty || b->shape_dirty) {
    int rc = build_groups(b, p, max_steps);
    if (rc != KR_OK) return rc;
  }
  if (p.n_groups == 0) return KR_OK;
  cudaStream_t st = part_stream(b, p);
  BatchArgs A{};
  A.K = b->K;
  A.tpl = b->d_tpl;
  A.T = b->T;
  A.state = b->d_state; A.grip = b->d_grip; A.glam = b->d_glam; A.cd = b->d_cd; A.ctrl_cur = b->d_ctrl; A.meta = b->d_meta;
  A.rects = b->d_rects; A.map_off = b->d_map_off; A.map_cull = b->d_map_cull;
  A.groups = p.d_groups; A.n_groups = p.n_groups; A.cpc = b->cpc; A.queue = p.d_queue;
  A.max_steps = max_steps;
  A.stop = p.stop;
  A.tag_done = p.tag_done;
  A.ctrl_period = std::max(1, b->d.control_period);
  A.obs = b->d_obs; A.obs_ring = b->d.obs_ring;
  A.slip_max = b->d.grip_slip_max; A.cooldown = b->d.grip_cooldown;
  A.inv_h64 = 1.0 / b->d.solver.h;
  A.dt = b->d.solver.h * b->d.solver.substeps;
  A.h64 = b->d.solver.h;
  A.substeps = b->d.solver.substeps;
  A.pw = b->d_pw; A.pw_idx = b->d_pw_idx; A.pw_stride = b->pw_stride;
  A.net = b->d_net; A.rects64 = b->d_rects64; A.lights = b->d_lights; A.light_off = b->d_light_off;
  A.map_size = b->d_map_size;
  A.light_tab = b->d_light_tab; A.light_T = b->light_T;
  cudaError_t e;
  if ((e = cudaMemsetAsync(p.d_queue, 0, sizeof(int), st)) != cudaSuccess) return b->cuda_fail(e, "queue reset");
  if (timed) cudaEventRecord(p.ev0, st);
  int grid = 0;
  e = b->G == 32 ? launch_g<32>(A, b, st, p.n_groups, &grid)
                 : b->G == 16 ? launch_g<16>(A, b, st, p.n_groups, &grid) : launch_g<8>(A, b, st, p.n_groups, &grid);
  if (e != cudaSuccess) return b->cuda_fail(e, "batch_kernel launch");
  if (grid == 0) return b->fail(KR_ERR_CAPACITY, "batch kernel does not fit on an SM with this launch shape");
  if (timed) cudaEventRecord(p.ev1, st);
  // remaining horizons as the next schedule sees them
  if (p.all) {
    for (int s = 0; s < b->capacity; s++)
      if (b->h_remaining[s] > 0) b->h_remaining[s] = std::max(0, b->h_remaining[s] - max_steps);
  } else {
    for (int s : p.slots)
      if (b->h_remaining[s] > 0) b->h_remaining[s] = std::max(0, b->h_remaining[s] - max_steps);
  }
  return KR_OK;
}

int prepare_spawn_into(kr_batch *b, int n, const int32_t *arms, const int32_t *segs, const int32_t *map_id,
                       const double *x, const double *y, const double *angle, const int32_t *horizon,
                       const uint32_t *control_seed, const float *tone, int ctrl_mode, const int32_t *ctrl,
                       float *pose, SlotMeta *meta, int *first_bad) {
  // checks and body templates, in order (a template is built on first use)
  const size_t tpl_before = b->tpls.size();
  std::vector<int> tid(n);
  for (int i = 0; i < n; i++) {
    *first_bad = i;
    const int t = ensure_template(b, arms[i], segs[i]);
    if (t < 0)
      return b->fail(KR_ERR_INVALID, "body shape " + std::to_string(arms[i]) + "x" + std::to_string(segs[i]) +
                                         " outside 1..8 arms x 1..9 segments");
    if (map_id[i] < 0 || map_id[i] >= b->n_maps)
      return b->fail(KR_ERR_INDEX, "map " + std::to_string(map_id[i]) + " of " + std::to_string(b->n_maps));
    if (horizon[i] < 0) return b->fail(KR_ERR_INVALID, "negative horizon");
    tid[i] = t;
  }
  *first_bad = -1;
  // spawn poses (spawnKraken: a cos and a sin per segment, in f64) and slot
  // records of creatures [lo, hi); creatures are independent, so large
  // batches are split over host threads
  auto fill = [&](int lo, int hi) {
    double px[kr::kMaxTplBodies], py[kr::kMaxTplBodies], pa[kr::kMaxTplBodies];
    for (int i = lo; i < hi; i++) {
      const kr::Template &T = b->tpls[tid[i]];
      kr::spawn_pose(T, x[i], y[i], angle[i], 0.28, px, py, pa);
      float *dst = pose + (size_t)i * kStateStride;
      std::fill(dst, dst + kStateStride, 0.f);
      for (int j = 0; j < T.nb; j++) {
        dst[j] = (float)px[j];
        dst[kBodyPad + j] = (float)py[j];
        dst[4 * kBodyPad + j] = (float)pa[j];
      }
      SlotMeta &m = meta[i];
      m = SlotMeta{};
      m.tpl = tid[i];
      m.map = map_id[i];
      m.horizon = horizon[i];
      m.step = 0;
      m.ctrl = ctrl ? ctrl[i] : ctrl_mode;
      m.rng = control_seed ? control_seed[i] : 0u;
      const double tn = std::max(0.0, std::min(1.0, tone ? (double)tone[i] : 0.5));
      m.tone = (float)tn;
      m.comp = (float)(1.0 / (2000.0 + tn * (400000.0 - 2000.0)));
      m.last_x = (double)(float)x[i];
      m.last_y = (double)(float)y[i];
      m.tone_d = tn;
      m.spawn_x = x[i];
      m.spawn_y = y[i];
      m.spawn_reach = T.reach;  // replaced by measureReach in spawn_kernel
    }
  };
  constexpr int kPerThread = 1024;
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int nt = std::min({16, hw, n / kPerThread});
  if (nt <= 1) {
    fill(0, n);
  } else {
    std::vector<std::thread> th;
    int started = 0;
    for (int k = 1; k < nt; k++) {
      const int lo = (int)((long)n * k / nt), hi = (int)((long)n * (k + 1) / nt);
      try {
        th.emplace_back(fill, lo, hi);
        started = k;
      } catch (const std::system_error &) {
        break;  // no more threads: this thread fills the rest
      }
    }
    fill(0, (int)((long)n * 1 / nt));
    if (started < nt - 1) fill((int)((long)n * (started + 1) / nt), n);
    for (auto &t : th) t.join();
  }
  if (b->tpls.size() != tpl_before) return upload_templates(b);
  return KR_OK;
}

int prepare_spawn(kr_batch *b, int n, const int32_t *arms, const int32_t *segs, const int32_t *map_id,
                  const double *x, const double *y, const double *angle, const int32_t *horizon,
                  const uint32_t *control_seed, const float *tone, int ctrl_mode, SpawnInit *out,
                  int *first_bad) {
  out->pose.resize((size_t)n * kStateStride);
  out->meta.resize(n);
  return prepare_spawn_into(b, n, arms, segs, map_id, x, y, angle, horizon, control_seed, tone, ctrl_mode, nullptr,
                            out->pose.data(), out->meta.data(), first_bad);
}

cudaError_t launch_spawn(kr_batch *b, const int *d_slots, const float *d_pose, const SlotMeta *d_meta,
                         int n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  spawn_kernel<<<n, 128, 0, stream>>>(b->d_state, b->d_grip, b->d_glam, b->d_cd, b->d_meta, b->d_ctrl,
                                      d_slots, d_pose, d_meta, n, b->d_rects64, b->d_map_off, b->rays,
                                      b->d_net, b->d_lights, b->d_light_off);
  return cudaGetLastError();
}

// kr_batch_run under time slices, every live slot to its horizon: launches
// preempted through the stop word after slice_ms, each followed by the
// step counters' readback and a regrouping of the creatures still live.
// The whole run's device time goes to the part's ev0 / ev1.
int run_sliced(kr_batch *b, int max_steps) {
  Part &p = b->main;
  cudaStream_t st = part_stream(b, p);
  cudaError_t e = cudaSuccess;
  if (!b->slice_ready) {
    if (!b->d_stop) e = cudaMalloc(&b->d_stop, sizeof(int));
    if (e == cudaSuccess && !b->h_flag) e = cudaMallocHost(&b->h_flag, 2 * sizeof(int));
    if (e == cudaSuccess && !b->d_steps) e = cudaMalloc(&b->d_steps, (size_t)b->capacity * sizeof(int));
    if (e == cudaSuccess && !b->h_steps) e = cudaMallocHost(&b->h_steps, (size_t)b->capacity * sizeof(int));
    if (e == cudaSuccess && !b->ctl) e = cudaStreamCreateWithFlags(&b->ctl, cudaStreamNonBlocking);
    if (e == cudaSuccess && !b->slice_start) e = cudaEventCreateWithFlags(&b->slice_start, cudaEventDisableTiming);
    if (e == cudaSuccess && !b->slice_end) e = cudaEventCreateWithFlags(&b->slice_end, cudaEventDisableTiming);
    if (e != cudaSuccess) return b->cuda_fail(e, "time-slice setup");
    b->h_flag[0] = 0;
    b->h_flag[1] = 1;
    b->slice_ready = true;
  }
  std::vector<int> run;  // the slots live when the run starts
  for (int s = 0; s < b->capacity; s++)
    if (b->h_remaining[s] > 0) run.push_back(s);
  using clk = std::chrono::steady_clock;
  double slice_s = b->slice_ms * 1e-3;
  long long steps_before = -1;
  b->last_slices = b->last_kernels = 0;
  b->last_creature_launches = 0;
  long live = (long)run.size();
  for (int k = 0;; k++) {
    e = cudaMemcpyAsync(b->d_stop, b->h_flag, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventRecord(b->slice_start, st);
    // the stop word's copy on the control stream comes after its reset
    if (e == cudaSuccess) e = cudaStreamWaitEvent(b->ctl, b->slice_start, 0);
    if (e != cudaSuccess) return b->cuda_fail(e, "slice start");
    p.stop = b->d_stop;
    p.dirty = true;
    int rc = launch_part(b, p, max_steps, k == 0);
    p.stop = nullptr;
    if (rc != KR_OK) return rc;
    if (p.n_groups == 0) break;
    b->last_slices++;
    b->last_kernels++;
    b->last_creature_launches += live;
    e = cudaEventRecord(b->slice_end, st);
    if (e != cudaSuccess) return b->cuda_fail(e, "slice record");
    // the slice's time counts from when its launch is next on the stream
    bool started = false, stopped = false;
    clk::time_point t0{};
    for (;;) {
      e = cudaEventQuery(b->slice_end);
      if (e == cudaSuccess) break;
      if (e != cudaErrorNotReady) return b->cuda_fail(e, "slice query");
      if (!started) {
        const cudaError_t q = cudaEventQuery(b->slice_start);
        if (q == cudaSuccess) {
          started = true;
          t0 = clk::now();
        } else if (q != cudaErrorNotReady) {
          return b->cuda_fail(q, "slice query");
        }
      } else if (!stopped && std::chrono::duration<double>(clk::now() - t0).count() >= slice_s) {
        e = cudaMemcpyAsync(b->d_stop, b->h_flag + 1, sizeof(int), cudaMemcpyHostToDevice, b->ctl);
        if (e != cudaSuccess) return b->cuda_fail(e, "slice stop");
        stopped = true;
      }
      std::this_thread::sleep_for(std::chrono::microseconds(20));
    }
    // the stop word's copy has landed before the next slice resets it
    if (stopped && (e = cudaStreamSynchronize(b->ctl)) != cudaSuccess) return b->cuda_fail(e, "slice stop wait");
    if (!stopped) break;  // every creature reached its horizon inside the slice
    step_counts_kernel<<<(b->capacity + 255) / 256, 256, 0, st>>>(b->d_meta, b->capacity, b->d_steps);
    b->last_kernels++;
    e = cudaGetLastError();
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(b->h_steps, b->d_steps, (size_t)b->capacity * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return b->cuda_fail(e, "slice step counters");
    live = 0;
    long long steps = 0;
    for (int s : run) {
      b->h_remaining[s] = std::max(0, b->h_meta[s].horizon - b->h_steps[s]);
      live += b->h_remaining[s] > 0;
      steps += b->h_steps[s];
    }
    if (live == 0) break;
    if (steps == steps_before) slice_s *= 2;  // no creature advanced: a longer slice
    steps_before = steps;
  }
  if (b->last_slices > 0 && (e = cudaEventRecord(p.ev1, st)) != cudaSuccess) return b->cuda_fail(e, "slice timing");
  return KR_OK;
}

}  // namespace krb

using namespace krb;

extern "C" const char *kr_batch_last_error(const kr_batch *b) {
  return b ? b->err.c_str() : g_batch_error.c_str();
}

extern "C" int kr_batch_create(const kr_batch_desc *desc, kr_batch **out) {
  if (!desc || !out) { g_batch_error = "kr_batch_create: null argument"; return KR_ERR_INVALID; }
  *out = nullptr;
  const kr_batch_desc &d = *desc;
  const kr_solver_params &p = d.solver;
  const float hf = (float)p.h;
  if (!(p.iterations >= 1 && p.iterations <= 64) || !(p.substeps >= 1 && p.substeps <= 64) ||
      !(hf > 0.f && hf < 1.f)) {
    g_batch_error = "implausible solver parameters (iterations 1..64, substeps 1..64, 0 < h < 1)";
    return KR_ERR_INVALID;
  }
  if (d.n_maps < 1 || !d.rects || !d.map_rect_off) { g_batch_error = "need at least one map"; return KR_ERR_INVALID; }
  if (d.capacity < 1 || d.capacity > (1 << 24)) { g_batch_error = "capacity out of range"; return KR_ERR_INVALID; }
  if (d.obs_ring < 0 || d.obs_ring > 4096) { g_batch_error = "obs_ring out of range 0..4096"; return KR_ERR_INVALID; }
  if (d.control_mode < 0 || d.control_mode > KR_CTRL_NET) { g_batch_error = "unknown control mode"; return KR_ERR_INVALID; }
  if (d.control_mode == KR_CTRL_NET && d.lights) {
    if (!d.map_light_off || !d.map_size) { g_batch_error = "lights without map_light_off / map_size"; return KR_ERR_INVALID; }
    for (int m = 0; m < d.n_maps; m++) {
      const int n = d.map_light_off[m + 1] - d.map_light_off[m];
      if (d.map_light_off[m] < 0 || n < 0 || n > KR_NET_MAX_LIGHTS) {
        g_batch_error = "map " + std::to_string(m) + ": " + std::to_string(n) + " lights (0.." +
                        std::to_string(KR_NET_MAX_LIGHTS) + ")";
        return KR_ERR_INVALID;
      }
      for (int l = d.map_light_off[m]; l < d.map_light_off[m + 1]; l++)
        if (!(d.lights[6 * (size_t)l + 2] > 0)) {
          g_batch_error = "map " + std::to_string(m) + ": light radius must be positive";
          return KR_ERR_INVALID;
        }
    }
  }
  if (d.control_mode == KR_CTRL_STREAM && d.control_period < 1) { g_batch_error = "control_period < 1"; return KR_ERR_INVALID; }
  for (int m = 0; m < d.n_maps; m++) {
    const int n = d.map_rect_off[m + 1] - d.map_rect_off[m];
    if (d.map_rect_off[m] < 0 || !(n >= 1 && n <= 100000)) {
      g_batch_error = "map " + std::to_string(m) + ": nRects implausible: " + std::to_string(n);
      return KR_ERR_INVALID;
    }
  }
  int dev = 0, n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
    cudaGetLastError();
    g_batch_error = "no CUDA device available";
    return KR_ERR_NODEVICE;
  }
  kr_batch *b = new kr_batch();
  b->d = d;
  b->d.rects = nullptr;
  b->d.map_rect_off = nullptr;
  b->d.lights = nullptr;
  b->d.map_light_off = nullptr;
  b->d.map_size = nullptr;
  b->capacity = d.capacity;
  b->n_maps = d.n_maps;
  kr::SolverConsts &K = b->K;
  K.h = hf;
  K.invH = (float)(1.0 / p.h);
  K.invH2 = (float)(1.0 / (p.h * p.h));
  const float nl = -(float)p.lin_drag, na = -(float)p.ang_drag;
  K.linDamp = (float)std::exp((double)(nl * hf));
  K.angDamp = (float)std::exp((double)(na * hf));
  K.maxSpeed = (float)p.max_speed;
  K.maxAngSpeed = (float)p.max_ang_speed;
  K.substeps = p.substeps;
  K.iterations = p.iterations;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&b->smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&b->smem_reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  cudaDeviceGetAttribute(&b->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  auto bail = [&](cudaError_t e, const char *what) {
    g_batch_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    kr_batch_destroy(b);
    return KR_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) return bail(e, "cudaStreamCreate");
  b->own_stream = true;
  // maps: rects as x y x+w y+h, per-map culling distance (see kr_solver.cuh)
  const int n_rects = d.map_rect_off[d.n_maps];
  std::vector<float4> r4(n_rects);
  std::vector<int> off(d.map_rect_off, d.map_rect_off + d.n_maps + 1);
  b->h_map_cull.assign(d.n_maps, 0.f);
  for (int m = 0; m < d.n_maps; m++) {
    double ht = 0.0;
    for (int i = off[m]; i < off[m + 1]; i++) {
      const float x = d.rects[4 * i], y = d.rects[4 * i + 1], w = d.rects[4 * i + 2], h = d.rects[4 * i + 3];
      r4[i] = make_float4(x, y, x + w, y + h);
      const double t = 0.5 * std::min(std::fabs((double)w), std::fabs((double)h));
      ht = std::isfinite(t) ? std::max(ht, t) : HUGE_VAL;
    }
    const double c = ht + 2.0 + kr::kCullSlack + 1.0;
    b->h_map_cull[m] = std::isfinite(c) && c < 1e30 ? (float)c : 1e30f;
  }
  b->h_rects.assign(d.rects, d.rects + 4 * (size_t)n_rects);
  b->h_map_off = off;
  if ((e = upload_vec(&b->d_rects, r4)) != cudaSuccess) return bail(e, "upload(rects)");
  if ((e = upload_vec(&b->d_map_off, off)) != cudaSuccess) return bail(e, "upload(map offsets)");
  if ((e = upload_vec(&b->d_rects64, b->h_rects)) != cudaSuccess) return bail(e, "upload(rects f64)");
  for (int k = 0; k < 16; k++) {
    const double a = ((double)k / 16) * 3.141592653589793 * 2;
    b->rays.c[k] = std::cos(a);
    b->rays.s[k] = std::sin(a);
  }
  if ((e = upload_vec(&b->d_map_cull, b->h_map_cull)) != cudaSuccess) return bail(e, "upload(map cull)");
  const size_t C = (size_t)d.capacity;
  if ((e = cudaMalloc(&b->d_state, C * kStateStride * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc(state)");
  if ((e = cudaMalloc(&b->d_grip, C * KR_BATCH_MAX_ARMS * sizeof(float4))) != cudaSuccess) return bail(e, "cudaMalloc(grips)");
  if ((e = cudaMalloc(&b->d_glam, C * KR_BATCH_MAX_ARMS * sizeof(float2))) != cudaSuccess) return bail(e, "cudaMalloc(grip lambda)");
  if ((e = cudaMalloc(&b->d_cd, C * KR_BATCH_MAX_ARMS * sizeof(double2))) != cudaSuccess) return bail(e, "cudaMalloc(cooldown)");
  if ((e = cudaMalloc(&b->d_ctrl, C * kCtrlStride * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc(controls)");
  if ((e = cudaMemset(b->d_ctrl, 0, C * kCtrlStride * sizeof(float))) != cudaSuccess) return bail(e, "cudaMemset(controls)");
  if ((e = cudaMalloc(&b->d_meta, C * sizeof(SlotMeta))) != cudaSuccess) return bail(e, "cudaMalloc(meta)");
  if ((e = cudaMemset(b->d_meta, 0, C * sizeof(SlotMeta))) != cudaSuccess) return bail(e, "cudaMemset(meta)");
  if (d.obs_ring > 0) {
    if ((e = cudaMalloc(&b->d_obs, C * d.obs_ring * KR_OBS_STRIDE * sizeof(float))) != cudaSuccess) return bail(e, "cudaMalloc(obs)");
    if ((e = cudaMemset(b->d_obs, 0, C * d.obs_ring * KR_OBS_STRIDE * sizeof(float))) != cudaSuccess) return bail(e, "cudaMemset(obs)");
  }
  if (d.control_mode == KR_CTRL_NET) {
    if ((e = cudaMalloc(&b->d_net, C * sizeof(NetRec))) != cudaSuccess) return bail(e, "cudaMalloc(net records)");
    if ((e = cudaMemset(b->d_net, 0, C * sizeof(NetRec))) != cudaSuccess) return bail(e, "cudaMemset(net records)");
    if (d.lights) {
      const int nl = d.map_light_off[d.n_maps];
      std::vector<double> lv(d.lights, d.lights + 6 * (size_t)nl);
      std::vector<int> lo(d.map_light_off, d.map_light_off + d.n_maps + 1);
      std::vector<double> ms(d.map_size, d.map_size + 2 * (size_t)d.n_maps);
      if ((e = upload_vec(&b->d_lights, lv)) != cudaSuccess) return bail(e, "upload(lights)");
      if ((e = upload_vec(&b->d_light_off, lo)) != cudaSuccess) return bail(e, "upload(light offsets)");
      if ((e = upload_vec(&b->d_map_size, ms)) != cudaSuccess) return bail(e, "upload(map sizes)");
      b->light_T = light_table_steps(nl);
      if (b->light_T > 0) {
        if ((e = cudaMalloc(&b->d_light_tab, (size_t)nl * b->light_T * sizeof(double2))) != cudaSuccess)
          return bail(e, "cudaMalloc(light table)");
        light_table_kernel<<<d.n_maps, 32>>>(b->d_lights, b->d_light_off, b->d_map_size,
                                             d.solver.h * d.solver.substeps, b->light_T, b->d_light_tab);
        if ((e = cudaGetLastError()) == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return bail(e, "light table");
      }
    }
  }
  b->h_meta.assign(C, SlotMeta{});
  b->h_remaining.assign(C, 0);
  // every slot starts empty (horizon 0)
  *out = b;
  return KR_OK;
}

extern "C" int kr_batch_spawn(kr_batch *b, int32_t first, int32_t n, const int32_t *arms,
                              const int32_t *segs, const int32_t *map_id, const double *x,
                              const double *y, const double *angle, const int32_t *horizon,
                              const uint32_t *control_seed, const float *tone) {
  if (!b) return KR_ERR_INVALID;
  if (n <= 0) return KR_OK;
  if (first < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "spawn range outside the slots");
  if (!arms || !segs || !map_id || !x || !y || !angle || !horizon)
    return b->fail(KR_ERR_INVALID, "kr_batch_spawn: null argument");
  std::vector<uint32_t> seeds(n);
  for (int i = 0; i < n; i++) seeds[i] = control_seed ? control_seed[i] : (uint32_t)(first + i);
  SpawnInit init;
  int bad = -1;
  int rc = prepare_spawn(b, n, arms, segs, map_id, x, y, angle, horizon, seeds.data(), tone,
                         b->d.control_mode, &init, &bad);
  if (rc != KR_OK) {
    b->err = "creature " + std::to_string(first + bad) + ": " + b->err;
    return rc;
  }
  std::vector<int> slots(n);
  for (int i = 0; i < n; i++) {
    slots[i] = first + i;
    b->h_meta[first + i] = init.meta[i];
    b->h_remaining[first + i] = init.meta[i].horizon;
  }
  float *d_pose = nullptr;
  SlotMeta *d_init = nullptr;
  int *d_slots = nullptr;
  cudaError_t e = cudaMallocAsync(&d_pose, init.pose.size() * sizeof(float), b->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_init, init.meta.size() * sizeof(SlotMeta), b->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(&d_slots, slots.size() * sizeof(int), b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_pose, init.pose.data(), init.pose.size() * sizeof(float), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_init, init.meta.data(), init.meta.size() * sizeof(SlotMeta), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_slots, slots.data(), slots.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = launch_spawn(b, d_slots, d_pose, d_init, n, b->stream);
  if (d_pose) cudaFreeAsync(d_pose, b->stream);
  if (d_init) cudaFreeAsync(d_init, b->stream);
  if (d_slots) cudaFreeAsync(d_slots, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_spawn");
  b->main.dirty = true;
  return KR_OK;
}

extern "C" int kr_batch_set_controls(kr_batch *b, const float *controls) {
  if (!b) return KR_ERR_INVALID;
  if (!controls) return b->fail(KR_ERR_INVALID, "kr_batch_set_controls: null buffer");
  cudaError_t e = cudaMemcpyAsync(b->d_ctrl, controls, (size_t)b->capacity * kCtrlStride * sizeof(float),
                                  cudaMemcpyHostToDevice, b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_set_controls");
  return KR_OK;
}

extern "C" int kr_batch_set_policy(kr_batch *b, const float *weights, int32_t n_individuals,
                                   int32_t n_params, const int32_t *slot_individual) {
  if (!b) return KR_ERR_INVALID;
  if (!weights || !slot_individual || n_individuals <= 0 || n_params <= 0)
    return b->fail(KR_ERR_INVALID, "kr_batch_set_policy: null argument or empty policy");
  // the body shape of every individual: the template of the live slots using it
  std::vector<int> ind_tpl(n_individuals, -1);
  for (int s = 0; s < b->capacity; s++) {
    if (slot_individual[s] < 0 || slot_individual[s] >= n_individuals)
      return b->fail(KR_ERR_INDEX, "slot " + std::to_string(s) + " refers to individual " +
                                       std::to_string(slot_individual[s]) + " of " +
                                       std::to_string(n_individuals));
    const SlotMeta &m = b->h_meta[s];
    if (m.horizon <= 0) continue;
    const kr::Template &t = b->tpls[m.tpl];
    const int need = policy_param_count(t.arms, t.segs);
    if (n_params < need)
      return b->fail(KR_ERR_INVALID, "slot " + std::to_string(s) + ": a " + std::to_string(t.arms) + "x" +
                                         std::to_string(t.segs) + " body needs " + std::to_string(need) +
                                         " policy parameters, got " + std::to_string(n_params));
    int &it = ind_tpl[slot_individual[s]];
    if (it >= 0 && it != m.tpl)
      return b->fail(KR_ERR_INVALID, "individual " + std::to_string(slot_individual[s]) +
                                         " is used by two body shapes");
    it = m.tpl;
  }
  const int stride = (n_params + 3) & ~3;  // 16-byte aligned individuals
  std::vector<float> dev((size_t)n_individuals * stride, 0.f);
  for (int k = 0; k < n_individuals; k++) {
    if (ind_tpl[k] < 0) continue;
    const kr::Template &t = b->tpls[ind_tpl[k]];
    transpose_policy(weights + (size_t)k * n_params, t.arms, t.segs, dev.data() + (size_t)k * stride);
  }
  const size_t need = dev.size();
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_set_policy sync");
  if (!b->d_pw || b->pw_capacity < need) {
    if (b->d_pw) cudaFree(b->d_pw);
    b->d_pw = nullptr;
    e = cudaMalloc(&b->d_pw, need * sizeof(float));
    if (e != cudaSuccess) return b->cuda_fail(e, "cudaMalloc(policy weights)");
    b->pw_capacity = need;
  }
  if (!b->d_pw_idx) {
    e = cudaMalloc(&b->d_pw_idx, (size_t)b->capacity * sizeof(int));
    if (e != cudaSuccess) return b->cuda_fail(e, "cudaMalloc(policy index)");
  }
  e = cudaMemcpyAsync(b->d_pw, dev.data(), need * sizeof(float), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_pw_idx, slot_individual, (size_t)b->capacity * sizeof(int),
                        cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_set_policy");
  b->n_individuals = n_individuals;
  b->pw_stride = stride;
  b->h_pw_idx.assign(slot_individual, slot_individual + b->capacity);
  b->h_pw_tpl = ind_tpl;
  return KR_OK;
}

// net.js's genome layout to the device layout (net_device_slots)
static void net_transpose(const float *w, int arms, float *dev) {
  const int n = net_param_count(arms);
  for (int p = 0; p < n; p++) {
    int d0 = 0, d1 = 0;
    const int k = net_device_slots(arms, p, &d0, &d1);
    if (k > 0) dev[d0] = w[p];
    if (k > 1) dev[d1] = w[p];
  }
}

extern "C" int kr_batch_set_net(kr_batch *b, const float *genomes, int32_t n_individuals, int32_t n_params,
                                const int32_t *slot_individual) {
  if (!b) return KR_ERR_INVALID;
  if (b->d.control_mode != KR_CTRL_NET) return b->fail(KR_ERR_STATE, "kr_batch_set_net on an engine without KR_CTRL_NET");
  if (!genomes || !slot_individual || n_individuals <= 0 || n_params <= 0)
    return b->fail(KR_ERR_INVALID, "kr_batch_set_net: null argument or empty genome set");
  // the arm count of every individual: that of the spawned slots using it
  std::vector<int> ind_arms(n_individuals, -1);
  for (int s = 0; s < b->capacity; s++) {
    if (slot_individual[s] < 0 || slot_individual[s] >= n_individuals)
      return b->fail(KR_ERR_INDEX, "slot " + std::to_string(s) + " refers to individual " +
                                       std::to_string(slot_individual[s]) + " of " + std::to_string(n_individuals));
    const SlotMeta &m = b->h_meta[s];
    if (m.horizon <= 0) continue;
    const int arms = b->tpls[m.tpl].arms, need = net_param_count(arms);
    if (n_params < need)
      return b->fail(KR_ERR_INVALID, "slot " + std::to_string(s) + ": a " + std::to_string(arms) +
                                         "-armed body's net has " + std::to_string(need) + " weights, got " +
                                         std::to_string(n_params));
    int &ia = ind_arms[slot_individual[s]];
    if (ia >= 0 && ia != arms)
      return b->fail(KR_ERR_INVALID, "individual " + std::to_string(slot_individual[s]) +
                                         " is used by two arm counts");
    ia = arms;
  }
  const int stride = (n_params + 3) & ~3;
  std::vector<float> dev((size_t)n_individuals * stride, 0.f);
  for (int k = 0; k < n_individuals; k++)
    if (ind_arms[k] >= 0) net_transpose(genomes + (size_t)k * n_params, ind_arms[k], dev.data() + (size_t)k * stride);
  const size_t need = dev.size();
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_set_net sync");
  if (!b->d_pw || b->pw_capacity < need) {
    if (b->d_pw) cudaFree(b->d_pw);
    b->d_pw = nullptr;
    e = cudaMalloc(&b->d_pw, need * sizeof(float));
    if (e != cudaSuccess) return b->cuda_fail(e, "cudaMalloc(genomes)");
    b->pw_capacity = need;
  }
  if (!b->d_pw_idx) {
    e = cudaMalloc(&b->d_pw_idx, (size_t)b->capacity * sizeof(int));
    if (e != cudaSuccess) return b->cuda_fail(e, "cudaMalloc(genome index)");
  }
  e = cudaMemcpyAsync(b->d_pw, dev.data(), need * sizeof(float), cudaMemcpyHostToDevice, b->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_pw_idx, slot_individual, (size_t)b->capacity * sizeof(int), cudaMemcpyHostToDevice,
                        b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_set_net");
  b->n_individuals = n_individuals;
  b->pw_stride = stride;
  b->h_pw_idx.assign(slot_individual, slot_individual + b->capacity);
  b->h_pw_arms = ind_arms;
  return KR_OK;
}

extern "C" int kr_batch_read_net(kr_batch *b, int32_t first, int32_t n, float *inputs, float *outputs) {
  if (!b) return KR_ERR_INVALID;
  if (!b->d_net) return b->fail(KR_ERR_STATE, "kr_batch_read_net on an engine without KR_CTRL_NET");
  if (first < 0 || n < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "read range outside the slots");
  if (n == 0) return KR_OK;
  const NetRec *src = b->d_net + first;
  cudaError_t e = cudaSuccess;
  if (inputs)
    e = cudaMemcpy2DAsync(inputs, KR_NET_IN_STRIDE * sizeof(float), src->x, sizeof(NetRec),
                          KR_NET_IN_STRIDE * sizeof(float), n, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess && outputs)
    e = cudaMemcpy2DAsync(outputs, KR_NET_OUT_STRIDE * sizeof(float), src->out, sizeof(NetRec),
                          KR_NET_OUT_STRIDE * sizeof(float), n, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_read_net");
  return KR_OK;
}

extern "C" int kr_batch_set_launch(kr_batch *b, int32_t lanes_per_creature, int32_t warps_per_cta,
                                   int32_t ctas_per_sm) {
  if (!b) return KR_ERR_INVALID;
  if (lanes_per_creature == 0) {  // back to the automatic shape of every launch
    if (!b->auto_shape || b->ctas_per_sm != 0) {
      b->main.dirty = true;
      b->shape_dirty = true;
    }
    b->ctas_per_sm = 0;
    b->auto_shape = true;
    return KR_OK;
  }
  if (lanes_per_creature != 32 && lanes_per_creature != 16 && lanes_per_creature != 8)
    return b->fail(KR_ERR_INVALID, "lanes_per_creature must be 32, 16 or 8 (0: automatic)");
  if (warps_per_cta < 1 || warps_per_cta > kMaxW) return b->fail(KR_ERR_INVALID, "warps_per_cta outside 1..16");
  if (warps_per_cta * (32 / lanes_per_creature) > kMaxCPC)
    return b->fail(KR_ERR_INVALID, "more than 64 creatures per CTA");
  if (ctas_per_sm < 0 || ctas_per_sm > 32) return b->fail(KR_ERR_INVALID, "ctas_per_sm outside 0..32");
  if (b->W != warps_per_cta || b->G != lanes_per_creature || b->ctas_per_sm != ctas_per_sm) {
    b->main.dirty = true;
    b->shape_dirty = true;
  }
  b->G = lanes_per_creature;
  b->W = warps_per_cta;
  b->ctas_per_sm = ctas_per_sm;
  b->auto_shape = false;
  return KR_OK;
}

extern "C" int kr_batch_set_unroll(kr_batch *b, int32_t substep_unroll) {
  if (!b) return KR_ERR_INVALID;
  if (substep_unroll != 1 && substep_unroll != 2) return b->fail(KR_ERR_INVALID, "substep_unroll must be 1 or 2");
  b->unroll = substep_unroll;
  return KR_OK;
}

extern "C" int kr_batch_get_unroll(kr_batch *b, int32_t *substep_unroll) {
  if (!b || !substep_unroll) return KR_ERR_INVALID;
  *substep_unroll = b->unroll;
  return KR_OK;
}

extern "C" int kr_batch_get_launch(kr_batch *b, int32_t *lanes_per_creature, int32_t *warps_per_cta,
                                   int32_t *ctas_per_sm, int32_t *smem_bytes) {
  if (!b) return KR_ERR_INVALID;
  if (b->shape_dirty && !b->h_tpl.empty()) {
    int rc = plan_shape(b);
    if (rc != KR_OK) return rc;
  }
  if (lanes_per_creature) *lanes_per_creature = b->G;
  if (warps_per_cta) *warps_per_cta = b->W;
  if (ctas_per_sm) *ctas_per_sm = b->ctas_per_sm;
  if (smem_bytes) *smem_bytes = (int32_t)b->smem_dyn;
  return KR_OK;
}

extern "C" int kr_batch_run(kr_batch *b, int32_t max_steps) {
  if (!b) return KR_ERR_INVALID;
  if (max_steps < 0) return b->fail(KR_ERR_INVALID, "max_steps < 0");
  if (max_steps == 0) return KR_OK;
  b->main.dirty = true;  // finished slots leave the queue, work estimates change
  if (b->slice_ms > 0.f) {
    bool to_horizon = true;
    for (int s = 0; s < b->capacity && to_horizon; s++) to_horizon = b->h_remaining[s] <= max_steps;
    if (to_horizon) return run_sliced(b, max_steps);
  }
  long long live = 0;
  for (int s = 0; s < b->capacity; s++) live += b->h_remaining[s] > 0;
  const int rc = launch_part(b, b->main, max_steps, true);
  b->last_slices = b->last_kernels = b->main.n_groups > 0 ? 1 : 0;
  b->last_creature_launches = b->main.n_groups > 0 ? live : 0;
  return rc;
}

extern "C" int kr_batch_set_slice(kr_batch *b, float slice_ms) {
  if (!b) return KR_ERR_INVALID;
  if (!(slice_ms >= 0.f && slice_ms < 1e7f)) return b->fail(KR_ERR_INVALID, "slice_ms outside [0, 1e7)");
  b->slice_ms = slice_ms;
  return KR_OK;
}

extern "C" int kr_batch_last_slices(kr_batch *b, int32_t *slices, int32_t *kernels, int64_t *creature_launches) {
  if (!b) return KR_ERR_INVALID;
  if (slices) *slices = b->last_slices;
  if (kernels) *kernels = b->last_kernels;
  if (creature_launches) *creature_launches = b->last_creature_launches;
  return KR_OK;
}

extern "C" int kr_batch_run_launches(kr_batch *b, int32_t steps_per_launch, int32_t launches) {
  if (!b) return KR_ERR_INVALID;
  if (steps_per_launch <= 0 || launches < 0) return b->fail(KR_ERR_INVALID, "kr_batch_run_launches: bad counts");
  b->main.dirty = true;
  for (int l = 0; l < launches; l++) {
    // the groups of the first launch serve every launch (finished slots are skipped by the kernel)
    int rc = launch_part(b, b->main, steps_per_launch, l == launches - 1);
    if (rc != KR_OK) return rc;
  }
  b->main.dirty = true;
  return KR_OK;
}

extern "C" int kr_batch_run_graph(kr_batch *b, int32_t max_steps, int32_t launches, int32_t replays) {
  if (!b) return KR_ERR_INVALID;
  if (max_steps <= 0 || launches <= 0 || replays < 0) return b->fail(KR_ERR_INVALID, "kr_batch_run_graph: bad counts");
  b->main.dirty = true;
  int rc = build_groups(b, b->main, max_steps);
  if (rc != KR_OK) return rc;
  if (b->main.staged_pending) {
    cudaEventSynchronize(b->main.staged);
    b->main.staged_pending = false;
  }
  const std::vector<int> before = b->h_remaining;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaStreamBeginCapture");
  for (int l = 0; l < launches && rc == KR_OK; l++) rc = launch_part(b, b->main, max_steps, false);
  e = cudaStreamEndCapture(b->stream, &graph);
  if (rc != KR_OK) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&exec, graph, 0);
  if (e != cudaSuccess) { cudaGraphDestroy(graph); return b->cuda_fail(e, "cudaGraphInstantiate"); }
  cudaEventRecord(b->main.ev0, b->stream);
  for (int r = 0; r < replays && e == cudaSuccess; r++) e = cudaGraphLaunch(exec, b->stream);
  cudaEventRecord(b->main.ev1, b->stream);
  cudaStreamSynchronize(b->stream);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaGraphLaunch");
  // every replay advanced every slot by launches x max_steps
  const long adv = (long)max_steps * launches * replays;
  for (int s = 0; s < b->capacity; s++) b->h_remaining[s] = (int)std::max<long>(0, before[s] - adv);
  b->main.dirty = true;
  return KR_OK;
}

extern "C" int kr_batch_autotune(kr_batch *b, int32_t steps, int32_t *lanes_out, int32_t *warps_out,
                                 int32_t *ctas_out, float *best_ms_out) {
  if (!b) return KR_ERR_INVALID;
  if (steps < 1) return b->fail(KR_ERR_INVALID, "autotune steps < 1");
  // (lanes per creature, warps per CTA, CTAs per SM, substep unroll)
  static const int kCand[][4] = {{8, 8, 0, 1},  {8, 16, 1, 1},  {8, 4, 4, 1},  {16, 8, 0, 1}, {16, 16, 1, 1},
                                 {32, 4, 0, 1}, {32, 8, 0, 1},  {8, 8, 0, 2},  {8, 16, 1, 2}, {16, 8, 0, 2},
                                 {32, 4, 0, 2}};
  const size_t C = (size_t)b->capacity;
  // scratch copy of every slot (the trials run, then the state goes back)
  float *t_state = nullptr, *t_ctrl = nullptr;
  float4 *t_grip = nullptr;
  float2 *t_glam = nullptr;
  double2 *t_cd = nullptr;
  SlotMeta *t_meta = nullptr;
  NetRec *t_net = nullptr;
  cudaError_t e = cudaMalloc(&t_state, C * kStateStride * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t_grip, C * KR_BATCH_MAX_ARMS * sizeof(float4));
  if (e == cudaSuccess) e = cudaMalloc(&t_glam, C * KR_BATCH_MAX_ARMS * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&t_cd, C * KR_BATCH_MAX_ARMS * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&t_ctrl, C * kCtrlStride * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&t_meta, C * sizeof(SlotMeta));
  if (e == cudaSuccess && b->d_net) e = cudaMalloc(&t_net, C * sizeof(NetRec));
  auto copy_slots = [&](bool save) {
    cudaError_t r = cudaSuccess;
    auto cp = [&](void *keep, void *live, size_t bytes) {
      if (r == cudaSuccess)
        r = cudaMemcpyAsync(save ? keep : live, save ? live : keep, bytes, cudaMemcpyDeviceToDevice, b->stream);
    };
    cp(t_state, b->d_state, C * kStateStride * sizeof(float));
    cp(t_grip, b->d_grip, C * KR_BATCH_MAX_ARMS * sizeof(float4));
    cp(t_glam, b->d_glam, C * KR_BATCH_MAX_ARMS * sizeof(float2));
    cp(t_cd, b->d_cd, C * KR_BATCH_MAX_ARMS * sizeof(double2));
    cp(t_ctrl, b->d_ctrl, C * kCtrlStride * sizeof(float));
    cp(t_meta, b->d_meta, C * sizeof(SlotMeta));
    if (b->d_net) cp(t_net, b->d_net, C * sizeof(NetRec));
    return r;
  };
  const std::vector<int> rem0 = b->h_remaining;
  const int G0 = b->G, W0 = b->W, C0 = b->ctas_per_sm, U0 = b->unroll;
  const bool auto0 = b->auto_shape;
  int best = -1, rc = KR_OK;
  float best_ms = 0.f;
  if (e == cudaSuccess) e = copy_slots(true);
  for (int c = 0; c < (int)(sizeof(kCand) / sizeof(kCand[0])) && e == cudaSuccess && rc == KR_OK; c++) {
    rc = kr_batch_set_launch(b, kCand[c][0], kCand[c][1], kCand[c][2]);
    if (rc != KR_OK) break;
    b->unroll = kCand[c][3];
    b->main.dirty = true;
    rc = launch_part(b, b->main, steps, true);
    if (rc == KR_ERR_CAPACITY) { rc = KR_OK; b->h_remaining = rem0; e = copy_slots(false); continue; }
    if (rc != KR_OK) break;
    float ms = 0.f;
    e = cudaEventSynchronize(b->main.ev1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->main.ev0, b->main.ev1);
    if (e == cudaSuccess && (best < 0 || ms < best_ms)) { best = c; best_ms = ms; }
    b->h_remaining = rem0;
    if (e == cudaSuccess) e = copy_slots(false);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFree(t_state); cudaFree(t_grip); cudaFree(t_glam); cudaFree(t_cd); cudaFree(t_ctrl); cudaFree(t_meta);
  if (t_net) cudaFree(t_net);
  b->h_remaining = rem0;
  b->main.dirty = true;
  if (rc != KR_OK) return rc;
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_autotune");
  if (best < 0) {  // nothing live: keep the shape as it was
    b->G = G0; b->W = W0; b->ctas_per_sm = C0; b->unroll = U0; b->auto_shape = auto0; b->shape_dirty = true;
  } else {
    rc = kr_batch_set_launch(b, kCand[best][0], kCand[best][1], kCand[best][2]);
    if (rc != KR_OK) return rc;
    b->unroll = kCand[best][3];
  }
  if (lanes_out) *lanes_out = b->G;
  if (warps_out) *warps_out = b->W;
  if (ctas_out) *ctas_out = b->ctas_per_sm;
  if (best_ms_out) *best_ms_out = best_ms;
  return KR_OK;
}

extern "C" int kr_batch_live(kr_batch *b, int32_t *live) {
  if (!b || !live) return KR_ERR_INVALID;
  std::vector<SlotMeta> m(b->capacity);
  cudaError_t e = cudaMemcpyAsync(m.data(), b->d_meta, m.size() * sizeof(SlotMeta), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_live");
  int n = 0;
  for (int s = 0; s < b->capacity; s++) {
    b->h_remaining[s] = std::max(0, m[s].horizon - m[s].step);
    if (b->h_remaining[s] > 0) n++;
  }
  *live = n;
  b->main.dirty = true;
  return KR_OK;
}

extern "C" int kr_batch_read_state(kr_batch *b, int32_t first, int32_t n, float *bodies, float *grips,
                                   int32_t *steps) {
  if (!b) return KR_ERR_INVALID;
  if (first < 0 || n < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "read range outside the slots");
  if (n == 0) return KR_OK;
  std::vector<float> st((size_t)n * kStateStride);
  std::vector<float4> gr((size_t)n * KR_BATCH_MAX_ARMS);
  std::vector<SlotMeta> m(n);
  cudaError_t e = cudaMemcpyAsync(st.data(), b->d_state + (size_t)first * kStateStride, st.size() * sizeof(float), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(gr.data(), b->d_grip + (size_t)first * KR_BATCH_MAX_ARMS, gr.size() * sizeof(float4), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(m.data(), b->d_meta + first, m.size() * sizeof(SlotMeta), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_read_state");
  constexpr int NB = kr::kMaxTplBodies;
  for (int i = 0; i < n; i++) {
    if (bodies)
      for (int j = 0; j < NB; j++)
        for (int f = 0; f < 6; f++) bodies[((size_t)i * NB + j) * 6 + f] = st[(size_t)i * kStateStride + f * kBodyPad + j];
    if (grips)
      for (int a = 0; a < KR_BATCH_MAX_ARMS; a++) {
        const float4 g = gr[(size_t)i * KR_BATCH_MAX_ARMS + a];
        float *o = grips + ((size_t)i * KR_BATCH_MAX_ARMS + a) * 4;
        o[0] = g.x; o[1] = g.y; o[2] = g.z; o[3] = g.w;
      }
    if (steps) steps[i] = m[i].step;
  }
  return KR_OK;
}

extern "C" int kr_batch_read_obs(kr_batch *b, int32_t first, int32_t n, float *obs) {
  if (!b || !obs) return KR_ERR_INVALID;
  if (b->d.obs_ring <= 0) return b->fail(KR_ERR_STATE, "no observation ring (obs_ring == 0)");
  if (first < 0 || n < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "read range outside the slots");
  const size_t per = (size_t)b->d.obs_ring * KR_OBS_STRIDE;
  cudaError_t e = cudaMemcpyAsync(obs, b->d_obs + (size_t)first * per, (size_t)n * per * sizeof(float),
                                  cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_read_obs");
  return KR_OK;
}

extern "C" int kr_batch_read_controls(kr_batch *b, int32_t first, int32_t n, float *controls) {
  if (!b || !controls) return KR_ERR_INVALID;
  if (first < 0 || n < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "read range outside the slots");
  cudaError_t e = cudaMemcpyAsync(controls, b->d_ctrl + (size_t)first * kCtrlStride,
                                  (size_t)n * kCtrlStride * sizeof(float), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_read_controls");
  return KR_OK;
}

extern "C" int kr_batch_read_fitness(kr_batch *b, int32_t first, int32_t n, double *out) {
  if (!b || !out) return KR_ERR_INVALID;
  if (first < 0 || n < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "read range outside the slots");
  std::vector<SlotMeta> m(n);
  cudaError_t e = cudaMemcpyAsync(m.data(), b->d_meta + first, m.size() * sizeof(SlotMeta), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_read_fitness");
  for (int i = 0; i < n; i++) {
    out[4 * i] = m[i].path_len; out[4 * i + 1] = m[i].last_x; out[4 * i + 2] = m[i].last_y;
    out[4 * i + 3] = m[i].attach_events;
  }
  return KR_OK;
}

extern "C" int kr_batch_read_metrics(kr_batch *b, int32_t first, int32_t n, double *out) {
  if (!b || !out) return KR_ERR_INVALID;
  if (first < 0 || n < 0 || first + n > b->capacity) return b->fail(KR_ERR_INVALID, "read range outside the slots");
  std::vector<SlotMeta> m(n);
  cudaError_t e = cudaMemcpyAsync(m.data(), b->d_meta + first, m.size() * sizeof(SlotMeta), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_read_metrics");
  for (int i = 0; i < n; i++) slot_metrics(m[i], out + (size_t)i * KR_METRIC_WORDS);
  return KR_OK;
}

extern "C" int kr_batch_last_ms(kr_batch *b, float *ms) {
  if (!b || !ms) return KR_ERR_INVALID;
  if (!b->main.ev1) return b->fail(KR_ERR_STATE, "no launch yet");
  cudaError_t e = cudaEventSynchronize(b->main.ev1);
  if (e == cudaSuccess) e = cudaEventElapsedTime(ms, b->main.ev0, b->main.ev1);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_last_ms");
  return KR_OK;
}

extern "C" int kr_batch_sync(kr_batch *b) {
  if (!b) return KR_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaStreamSynchronize");
  return KR_OK;
}

extern "C" int kr_batch_set_stream(kr_batch *b, void *stream) {
  if (!b) return KR_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "cudaStreamSynchronize");
  if (stream) {
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->own_stream = false;
    b->stream = static_cast<cudaStream_t>(stream);
  } else if (!b->own_stream) {
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
      return b->cuda_fail(e, "cudaStreamCreate");
    b->own_stream = true;
  }
  return KR_OK;
}

extern "C" void kr_batch_destroy(kr_batch *b) {
  if (!b) return;
  cudaDeviceSynchronize();
  for (void *p : b->d_tpl_arrays)
    if (p) cudaFree(p);
  free_part(b->main);
  void *ptrs[] = {b->d_tpl, const_cast<int *>(b->T.arm_segs), b->d_rects, b->d_map_off, b->d_map_cull, b->d_rects64,
                  b->d_state, b->d_grip, b->d_glam, b->d_cd, b->d_ctrl, b->d_meta, b->d_obs,
                  b->d_pw, b->d_pw_idx, b->s_state, b->s_grip, b->s_glam, b->s_cd,
                  b->s_ctrl, b->s_meta, b->s_groups, b->d_net, b->s_net, b->d_lights, b->d_light_off,
                  b->d_map_size, b->d_light_tab, b->d_stop, b->d_steps};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (b->h_flag) cudaFreeHost(b->h_flag);
  if (b->h_steps) cudaFreeHost(b->h_steps);
  if (b->ctl) cudaStreamDestroy(b->ctl);
  if (b->slice_start) cudaEventDestroy(b->slice_start);
  if (b->slice_end) cudaEventDestroy(b->slice_end);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

namespace {
template <typename T>
cudaError_t copy_all(T **dst, const T *src, size_t n, cudaStream_t st) {
  if (!*dst) {
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dst), n * sizeof(T));
    if (e != cudaSuccess) return e;
  }
  return cudaMemcpyAsync(*dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, st);
}
}  // namespace

extern "C" int kr_batch_snapshot(kr_batch *b) {
  if (!b) return KR_ERR_INVALID;
  const size_t C = (size_t)b->capacity;
  cudaError_t e = copy_all(&b->s_state, b->d_state, C * kStateStride, b->stream);
  if (e == cudaSuccess) e = copy_all(&b->s_grip, b->d_grip, C * KR_BATCH_MAX_ARMS, b->stream);
  if (e == cudaSuccess) e = copy_all(&b->s_glam, b->d_glam, C * KR_BATCH_MAX_ARMS, b->stream);
  if (e == cudaSuccess) e = copy_all(&b->s_cd, b->d_cd, C * KR_BATCH_MAX_ARMS, b->stream);
  if (e == cudaSuccess) e = copy_all(&b->s_ctrl, b->d_ctrl, C * kCtrlStride, b->stream);
  if (e == cudaSuccess) e = copy_all(&b->s_meta, b->d_meta, C, b->stream);
  if (e == cudaSuccess && b->d_net) e = copy_all(&b->s_net, b->d_net, C, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_snapshot");
  b->s_remaining = b->h_remaining;
  b->s_n_groups = -1;  // groups for this state are cached at the first restore
  return KR_OK;
}

extern "C" int kr_batch_restore(kr_batch *b) {
  if (!b) return KR_ERR_INVALID;
  if (!b->s_state) return b->fail(KR_ERR_STATE, "restore before snapshot");
  const size_t C = (size_t)b->capacity;
  cudaError_t e = cudaMemcpyAsync(b->d_state, b->s_state, C * kStateStride * sizeof(float), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_grip, b->s_grip, C * KR_BATCH_MAX_ARMS * sizeof(float4), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_glam, b->s_glam, C * KR_BATCH_MAX_ARMS * sizeof(float2), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_cd, b->s_cd, C * KR_BATCH_MAX_ARMS * sizeof(double2), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_ctrl, b->s_ctrl, C * kCtrlStride * sizeof(float), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(b->d_meta, b->s_meta, C * sizeof(SlotMeta), cudaMemcpyDeviceToDevice, b->stream);
  if (e == cudaSuccess && b->d_net && b->s_net)
    e = cudaMemcpyAsync(b->d_net, b->s_net, C * sizeof(NetRec), cudaMemcpyDeviceToDevice, b->stream);
  if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_restore");
  b->h_remaining = b->s_remaining;
  // the work groups of the snapshot state: built once, then copied back
  Part &p = b->main;
  if (b->s_n_groups < 0 || b->s_cpc != b->cpc || b->s_G != b->G || b->shape_dirty) {
    int rc = build_groups(b, p, 1 << 30);
    if (rc != KR_OK) return rc;
    if (b->s_groups) cudaFree(b->s_groups);
    b->s_groups = nullptr;
    e = cudaMalloc(&b->s_groups, std::max<size_t>(p.c_groups, 1) * sizeof(int));
    if (e == cudaSuccess && p.n_groups > 0)
      e = cudaMemcpyAsync(b->s_groups, p.d_groups, (size_t)p.n_groups * b->cpc * sizeof(int),
                          cudaMemcpyDeviceToDevice, b->stream);
    if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_restore(groups)");
    b->s_n_groups = p.n_groups;
    b->s_cpc = b->cpc;
    b->s_G = b->G;
  } else if (b->s_n_groups > 0) {
    e = cudaMemcpyAsync(p.d_groups, b->s_groups, (size_t)b->s_n_groups * b->cpc * sizeof(int),
                        cudaMemcpyDeviceToDevice, b->stream);
    if (e != cudaSuccess) return b->cuda_fail(e, "kr_batch_restore(groups)");
    p.n_groups = b->s_n_groups;
  }
  p.dirty = false;
  return KR_OK;
}

namespace {
// n independent f32 FMA chains per thread (no dependence between chains)
__global__ void fma_probe_kernel(float *out, int iters) {
  float a0 = threadIdx.x * 1e-3f, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
  float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
  const float m = 0.9999999f, c = 1e-7f;
  for (int i = 0; i < iters; i++) {
    a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
    a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
  }
  if (a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7 == 12345.f) out[threadIdx.x] = a0;
}
}  // namespace

namespace {
__global__ void sincos_probe_kernel(const float *x, int n, float *s, float *c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) kr::sincos_r(x[i], s + i, c + i);
}

__global__ void wrap_probe_kernel(const double *d, int n, double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = wrap_pi(d[i]);
}
}  // namespace

extern "C" int kr_probe_sincos(const float *x, int32_t n, float *s, float *c) {
  if (!x || !s || !c || n < 0) { g_batch_error = "kr_probe_sincos: bad arguments"; return KR_ERR_INVALID; }
  if (n == 0) return KR_OK;
  float *d = nullptr;
  cudaError_t e = cudaMalloc(&d, (size_t)n * 3 * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(d, x, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    sincos_probe_kernel<<<(n + 255) / 256, 256>>>(d, n, d + n, d + 2 * (size_t)n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(s, d + n, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(c, d + 2 * (size_t)n, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) { g_batch_error = cudaGetErrorString(e); return KR_ERR_CUDA; }
  return KR_OK;
}

extern "C" int kr_probe_wrap(const double *d, int32_t n, double *out) {
  if (!d || !out || n < 0) { g_batch_error = "kr_probe_wrap: bad arguments"; return KR_ERR_INVALID; }
  if (n == 0) return KR_OK;
  double *buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, (size_t)n * 2 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(buf, d, (size_t)n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    wrap_probe_kernel<<<(n + 255) / 256, 256>>>(buf, n, buf + n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, buf + n, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(buf);
  if (e != cudaSuccess) { g_batch_error = cudaGetErrorString(e); return KR_ERR_CUDA; }
  return KR_OK;
}

extern "C" int kr_probe_fp32_rate(double *fma_per_s) {
  if (!fma_per_s) return KR_ERR_INVALID;
  int dev = 0, n_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  cudaEvent_t e0, e1;
  cudaError_t e = cudaMalloc(&out, 1024 * sizeof(float));
  if (e != cudaSuccess) { g_batch_error = cudaGetErrorString(e); return KR_ERR_CUDA; }
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 1 << 16, blocks = n_sm * 8, threads = 256;
  fma_probe_kernel<<<blocks, threads>>>(out, 256);
  cudaEventRecord(e0);
  fma_probe_kernel<<<blocks, threads>>>(out, iters);
  cudaEventRecord(e1);
  e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess) { g_batch_error = cudaGetErrorString(e); return KR_ERR_CUDA; }
  *fma_per_s = (double)blocks * threads * iters * 8.0 / (ms * 1e-3);
  return KR_OK;
}
