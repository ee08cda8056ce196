// kr_solver.cuh -- device side of the XPBD creature step (sm_100a).
//
// One connected component of the world (one creature, an "island") is
// advanced by one warp.  Its bodies and constraints are staged in shared
// memory for the whole launch; lanes split each constraint level and the
// per-body collision work.  Nothing in here touches global memory except the
// read-only rect list of the map.
//
// Arithmetic follows tools/f32solver.mjs operation by operation: every
// intermediate is rounded to f32 with a non-contracting intrinsic
// (__fadd_rn/__fsub_rn/__fmul_rn/__fdiv_rn/__fsqrt_rn never fuse into an FMA),
// sin/cos are the f64 functions rounded once to f32 (Math.fround(Math.cos(x))),
// and the WGSL `%` uses the exact truncated quotient (f32solver.mjs:36-51).
#pragma once
#include <cstdint>

namespace kr {

// solver.wgsl:81, 93-94 and f32solver.mjs:26-33, as f32
constexpr float kSlackPos = 0.002f;
constexpr float kSlackAng = 0.0002f;
constexpr float kTau = 6.28318530718f;
constexpr float kPi = 3.14159265359f;
constexpr float kEpsDet = 1e-12f;
constexpr float kEpsSdf = 1e-12f;
constexpr float kSdfInf = 1e30f;
constexpr float kSdfValid = 1e29f;

struct SolverConsts {
  float h, invH, invH2, linDamp, angDamp, maxSpeed, maxAngSpeed;
  int substeps, iterations;
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }

// Math.fround(Math.sin(x)) and Math.fround(Math.cos(x)) for an f32 argument:
// both evaluated in f64 and rounded once to f32.  For |x| <= 2^20 the f64
// value comes from a three-part Cody-Waite reduction by pi/32, a table of
// sin / cos at k pi/32 and short Taylor series on |r| <= pi/64, the table
// value plus a small correction; larger or non-finite arguments use CUDA's
// f64 sincos.  Either way the f64 result is within a few f64 ulp of the
// exact value (measured on 4e7 arguments up to 2^20 against long-double
// sin / cos: relative error below 3.6e-16), so its rounding to f32 is the
// correctly rounded f32 except within a few 2^-29 of a rounding midpoint --
// the same class as glibc's and V8's f64 sin/cos.
//
// sin and cos of k pi / 32, k = 0..63, each the correctly rounded f64
__device__ const double2 kSinCosTab[64] = {
    {0.0, 1.0},
    {0.0980171403295606, 0.9951847266721969},
    {0.19509032201612828, 0.9807852804032304},
    {0.2902846772544624, 0.9569403357322088},
    {0.3826834323650898, 0.9238795325112867},
    {0.47139673682599764, 0.881921264348355},
    {0.5555702330196022, 0.8314696123025452},
    {0.6343932841636455, 0.773010453362737},
    {0.7071067811865476, 0.7071067811865476},
    {0.773010453362737, 0.6343932841636455},
    {0.8314696123025452, 0.5555702330196022},
    {0.881921264348355, 0.47139673682599764},
    {0.9238795325112867, 0.3826834323650898},
    {0.9569403357322088, 0.2902846772544624},
    {0.9807852804032304, 0.19509032201612828},
    {0.9951847266721969, 0.0980171403295606},
    {1.0, 0.0},
    {0.9951847266721969, -0.0980171403295606},
    {0.9807852804032304, -0.19509032201612828},
    {0.9569403357322088, -0.2902846772544624},
    {0.9238795325112867, -0.3826834323650898},
    {0.881921264348355, -0.47139673682599764},
    {0.8314696123025452, -0.5555702330196022},
    {0.773010453362737, -0.6343932841636455},
    {0.7071067811865476, -0.7071067811865476},
    {0.6343932841636455, -0.773010453362737},
    {0.5555702330196022, -0.8314696123025452},
    {0.47139673682599764, -0.881921264348355},
    {0.3826834323650898, -0.9238795325112867},
    {0.2902846772544624, -0.9569403357322088},
    {0.19509032201612828, -0.9807852804032304},
    {0.0980171403295606, -0.9951847266721969},
    {0.0, -1.0},
    {-0.0980171403295606, -0.9951847266721969},
    {-0.19509032201612828, -0.9807852804032304},
    {-0.2902846772544624, -0.9569403357322088},
    {-0.3826834323650898, -0.9238795325112867},
    {-0.47139673682599764, -0.881921264348355},
    {-0.5555702330196022, -0.8314696123025452},
    {-0.6343932841636455, -0.773010453362737},
    {-0.7071067811865476, -0.7071067811865476},
    {-0.773010453362737, -0.6343932841636455},
    {-0.8314696123025452, -0.5555702330196022},
    {-0.881921264348355, -0.47139673682599764},
    {-0.9238795325112867, -0.3826834323650898},
    {-0.9569403357322088, -0.2902846772544624},
    {-0.9807852804032304, -0.19509032201612828},
    {-0.9951847266721969, -0.0980171403295606},
    {-1.0, 0.0},
    {-0.9951847266721969, 0.0980171403295606},
    {-0.9807852804032304, 0.19509032201612828},
    {-0.9569403357322088, 0.2902846772544624},
    {-0.9238795325112867, 0.3826834323650898},
    {-0.881921264348355, 0.47139673682599764},
    {-0.8314696123025452, 0.5555702330196022},
    {-0.773010453362737, 0.6343932841636455},
    {-0.7071067811865476, 0.7071067811865476},
    {-0.6343932841636455, 0.773010453362737},
    {-0.5555702330196022, 0.8314696123025452},
    {-0.47139673682599764, 0.881921264348355},
    {-0.3826834323650898, 0.9238795325112867},
    {-0.2902846772544624, 0.9569403357322088},
    {-0.19509032201612828, 0.9807852804032304},
    {-0.0980171403295606, 0.9951847266721969}
};

// sin / cos beyond 2^20 and of non-finite arguments: CUDA's f64 sincos
// rounded to f32, out of line -- a cold path kept out of the instruction
// stream of the solve loops.
static __device__ __noinline__ float2 sincos_far(double x) {
  double sd, cd;
  sincos(x, &sd, &cd);
  return make_float2(static_cast<float>(sd), static_cast<float>(cd));
}

__device__ __forceinline__ void sincos_r(float a, float *s, float *c) {
  const double x = static_cast<double>(a);
  if (!(fabs(x) <= 1048576.0)) {
    const float2 f = sincos_far(x);
    *s = f.x;
    *c = f.y;
    return;
  }
  // x = k pi/32 + r, |r| <= pi/64: pi/32 in three parts (29, 29 and 53
  // bits), so k p1 and k p2 are exact for |k| < 2^24
  const double k = rint(x * 10.185916357881302);  // 32/pi
  double r = fma(-k, 0x1.921fb54000000p-4, x);
  r = fma(-k, 0x1.10b4611000000p-34, r);
  r = fma(-k, 0x1.4c4c6628b80dcp-63, r);
  const double r2 = r * r;
  // Taylor series on |r| <= pi/64: sin through r^7 (truncation below 5e-18
  // relative), cos - 1 through r^8 (below 3e-20)
  double ps = -1.0 / 5040;
  ps = fma(ps, r2, 1.0 / 120);
  ps = fma(ps, r2, -1.0 / 6);
  const double sr = fma(r * r2, ps, r);
  double pc = 1.0 / 40320;
  pc = fma(pc, r2, -1.0 / 720);
  pc = fma(pc, r2, 1.0 / 24);
  pc = fma(pc, r2, -0.5);
  const double cm1 = r2 * pc;                     // cos r - 1
  // sin(t + r) = S + (S (cos r - 1) + C sin r), cos(t + r) = C + (C (cos r - 1) - S sin r):
  // the table value plus a small correction
  const double2 t = __ldg(&kSinCosTab[static_cast<int>(static_cast<long long>(k) & 63)]);
  *s = static_cast<float>(t.x + fma(t.x, cm1, t.y * sr));
  *c = static_cast<float>(t.y + fma(t.y, cm1, -(t.x * sr)));
}

// trunc(x / TAU) exactly, as the f64 quotient of f32solver.mjs:38 gives it.
// The f32 estimate q = trunc(x * (1/TAU)) is off by at most one near an
// integer; the remainder x - q*TAU is then exact in one fma (both terms are
// multiples of 2^-21 for |x| >= 4 and it stays below 8 in magnitude) and
// decides the correction.  |x| < 4 has quotient 0.
__device__ __forceinline__ float trunc_quot_tau(float x) {
  if (fabsf(x) < 4.f) return 0.f;
  float q = truncf(__fmul_rn(x, 0.15915494f));
  const float r = fmaf(-q, kTau, x);
  if (x >= 0.f) {
    if (r < 0.f) q -= 1.f;
    else if (r >= kTau) q += 1.f;
  } else {
    if (r > 0.f) q += 1.f;
    else if (r <= -kTau) q -= 1.f;
  }
  return q;
}

// angleDeltaF, f32solver.mjs:36-43 (solver.wgsl:103-108)
__device__ __forceinline__ float angle_delta(float a, float b) {
  float x = fsub(a, b);
  float q = trunc_quot_tau(x);
  float d = fsub(x, fmul(kTau, q));
  if (d > kPi) return fsub(d, kTau);
  if (d < -kPi) return fadd(d, kTau);
  return d;
}

// wrapAngleF, f32solver.mjs:45-51 (solver.wgsl:96-101)
__device__ __forceinline__ float wrap_angle(float a) {
  float q = trunc_quot_tau(a);
  float d = fsub(a, fmul(kTau, q));
  if (d > kPi) return fsub(d, kTau);
  if (d < -kPi) return fadd(d, kTau);
  return d;
}

// lengthF, f32solver.mjs:54-56 (WGSL length(vec2f))
__device__ __forceinline__ float length2(float x, float y) {
  return fsqrt(fadd(fmul(x, x), fmul(y, y)));
}

// Rect as stored on the device: x, y, x + w, y + h (all f32, the sums
// rounded once as solver.wgsl:120-121 computes r.x + r.w).
// sdfF, f32solver.mjs:139-166 (solver.wgsl:114-147), over the rects
// idx[0..n) in ascending order (or 0..n when idx is null).  The division of
// the outward normal is deferred to the final winner: bnx/bny are overwritten
// by every later winner, so only the last winner's dx/best, dy/best survive.
__device__ __forceinline__ bool sdf(const float4 *__restrict__ rects, const short *idx, int n,
                                    float x, float y, float *od, float *onx, float *ony) {
  float best = kSdfInf, thr = __int_as_float(0x7f800000);  // f32 1e30*1e30 = +inf
  float wdx = 0.f, wdy = 0.f, inx = 0.f, iny = 0.f;
  bool inside = false;
  for (int q = 0; q < n; q++) {
    const float4 r = __ldg(rects + (idx ? idx[q] : q));
    float cx = x < r.x ? r.x : (x > r.z ? r.z : x);
    float cy = y < r.y ? r.y : (y > r.w ? r.w : y);
    float dx = fsub(x, cx), dy = fsub(y, cy);
    float d2 = fadd(fmul(dx, dx), fmul(dy, dy));
    if (d2 > kEpsSdf) {
      if (d2 < thr) {
        best = fsqrt(d2);
        thr = fmul(best, best);
        wdx = dx; wdy = dy;
        inside = false;
      }
    } else {
      float dl = fsub(x, r.x), dr = fsub(r.z, x), dt = fsub(y, r.y), db = fsub(r.w, y);
      float m = dl, nx = -1.f, ny = 0.f;
      if (dr < m) { m = dr; nx = 1.f; ny = 0.f; }
      if (dt < m) { m = dt; nx = 0.f; ny = -1.f; }
      if (db < m) { m = db; nx = 0.f; ny = 1.f; }
      float d = -m;
      if (d < best) {
        best = d;
        thr = fmul(best, best);
        inx = nx; iny = ny;
        inside = true;
      }
    }
  }
  if (best > kSdfValid) return false;
  *od = best;
  if (inside) { *onx = inx; *ony = iny; }
  else { *onx = fdiv(wdx, best); *ony = fdiv(wdy, best); }
  return true;
}

// Exact rect culling for one collision pass of one creature.
//
// Let D = max(largest collision radius, largest half-thickness min(w,h)/2 of
// a rect) + 2.  Drop every rect farther than D from every point the pass
// evaluates.  The sequential SDF fold then returns the same winner, or in
// both cases a winner farther than D - 1 (> radius + 1: no correction):
//  * a state's threshold f(best^2) never falls below the squared distance
//    of any rect processed so far, except that an inside winner sets it to
//    at most half-thickness^2 < (D - 1)^2; a dropped rect (d^2 > D^2) can
//    therefore only beat states with threshold >= (D - 1)^2 ("far" states);
//  * by monotone rounding, a rect that fails to beat a far state is itself
//    far, and an inside rect beats every far state; so the folds with and
//    without the dropped rects hold equal states or two far states.
// The pass keeps a point's evaluation on the culled list only while the
// point lies in the box the list was built for (kCullSlack inside the cull
// margin); otherwise it uses the full list.
constexpr int kMaxCulled = 64;
constexpr float kCullSlack = 6.f;

// A group of G lanes of one warp advancing one creature (G = 32, 16, 8):
// lanes of a group loop with stride G and synchronize, reduce and vote only
// among themselves, so a warp can carry 32 / G creatures of one template.
template <int G>
struct Lanes {
  int lane;        // 0 .. G-1
  int base;        // first warp lane of the group
  unsigned mask;   // the group's lanes in the warp
  __device__ __forceinline__ explicit Lanes(int warp_lane)
      : lane(warp_lane & (G - 1)), base(warp_lane & ~(G - 1)),
        mask(G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (warp_lane & ~(G - 1)))) {}
  __device__ __forceinline__ void sync() const { __syncwarp(mask); }
  __device__ __forceinline__ unsigned ballot(bool p) const {
    const unsigned b = __ballot_sync(mask, p);
    return G == 32 ? b : (b >> base) & ((1u << G) - 1u);
  }
  __device__ __forceinline__ float min(float v) const {
    for (int o = G / 2; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(mask, v, o, G));
    return v;
  }
  __device__ __forceinline__ float max(float v) const {
    for (int o = G / 2; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(mask, v, o, G));
    return v;
  }
};

// Shared-memory view of one island (one creature).  Constraint slots are in
// schedule order: level by level, each level body-disjoint.  Two layouts:
//  * per slot (gpuworld drop-in): every field an array over the slots;
//  * compact (batched engine): the template's statics, plus per creature
//    only lambda, the motor targets and the grip state (grips are the only
//    constraints with a moving anchor, a break force and a broken flag;
//    motors the only ones with a target and a nonzero compliance).
struct Island {
  // bodies (local index)
  float *px, *py, *ppx, *ppy, *vx, *vy, *ang, *angP, *av, *im, *ii, *fx, *fy, *tq;
  float *bs, *bc;  // sin / cos of angP during a collision pass
  // constraint slots
  const int *ab;   // a | (b << 16), b == 0xffff for a world anchor
  int *tb;         // per slot: type | (broken << 8)
  const float *lax, *lay, *rest, *minA, *maxA;
  float *lbx, *lby;         // per slot (drop-in); template statics (batched)
  float *comp, *tgt, *brk;  // per slot (drop-in)
  float *lamX, *lamY, *lam;
  // compact layout (batched engine)
  const int *type;   // per slot static type
  const int *garm;   // per slot: arm of a grip, else -1
  const int *motor;  // per slot: motor index of an angle constraint, else -1
  float *tgt_m;      // per motor target
  float *anc;        // per arm: anchor x, y, break force, broken (1.f / 0.f)
  float comp_m;      // motor compliance of the creature
  // collision points, grouped per local body in groupCollPoints order
  const float *plx, *ply, *pr;
  const int *pbody;       // local body of each point
  float *pdx, *pdy;       // speculative correction of each point
  int *pflag;             // 1 if the speculative evaluation corrects
  const int *boff, *bcnt;
  short *cull;            // culled rect list (kMaxCulled)
  int nb, nc, np, nlv;
  const int *lvl;         // level offsets, nlv + 1
};

// Field access of the two layouts (same values, different storage).
struct SlotAccess {
  __device__ static __forceinline__ int type(const Island &S, int k) { return S.tb[k] & 0xff; }
  __device__ static __forceinline__ bool broken(const Island &S, int k) { return (S.tb[k] >> 8) != 0; }
  __device__ static __forceinline__ void set_broken(Island &S, int k) { S.tb[k] |= 1 << 8; }
  __device__ static __forceinline__ float lbx(const Island &S, int k) { return S.lbx[k]; }
  __device__ static __forceinline__ float lby(const Island &S, int k) { return S.lby[k]; }
  __device__ static __forceinline__ float comp(const Island &S, int k) { return S.comp[k]; }
  __device__ static __forceinline__ float tgt(const Island &S, int k) { return S.tgt[k]; }
  __device__ static __forceinline__ float brk(const Island &S, int k) { return S.brk[k]; }
};
struct CompactAccess {
  __device__ static __forceinline__ int type(const Island &S, int k) { return S.type[k]; }
  __device__ static __forceinline__ bool broken(const Island &S, int k) {
    const int a = S.garm[k];
    return a >= 0 && S.anc[4 * a + 3] != 0.f;
  }
  __device__ static __forceinline__ void set_broken(Island &S, int k) { S.anc[4 * S.garm[k] + 3] = 1.f; }
  __device__ static __forceinline__ float lbx(const Island &S, int k) {
    const int a = S.garm[k];
    return a >= 0 ? S.anc[4 * a] : S.lbx[k];
  }
  __device__ static __forceinline__ float lby(const Island &S, int k) {
    const int a = S.garm[k];
    return a >= 0 ? S.anc[4 * a + 1] : S.lby[k];
  }
  __device__ static __forceinline__ float comp(const Island &S, int k) {
    return S.type[k] == 1 ? S.comp_m : 0.f;
  }
  __device__ static __forceinline__ float tgt(const Island &S, int k) { return S.tgt_m[S.motor[k]]; }
  __device__ static __forceinline__ float brk(const Island &S, int k) { return S.anc[4 * S.garm[k] + 2]; }
};

// integrateF, f32solver.mjs:177-200 (solver.wgsl:166-205)
__device__ __forceinline__ void integrate_body(const SolverConsts &K, Island &S, int i) {
  float im = S.im[i], ii = S.ii[i];
  if (im == 0.f && ii == 0.f) {
    S.ppx[i] = S.px[i]; S.ppy[i] = S.py[i]; S.angP[i] = S.ang[i];
    S.vx[i] = 0.f; S.vy[i] = 0.f; S.av[i] = 0.f;
    return;
  }
  float vx = fmul(fadd(S.vx[i], fmul(fmul(K.h, im), S.fx[i])), K.linDamp);
  float vy = fmul(fadd(S.vy[i], fmul(fmul(K.h, im), S.fy[i])), K.linDamp);
  float av = fmul(fadd(S.av[i], fmul(fmul(K.h, ii), S.tq[i])), K.angDamp);
  float sp = length2(vx, vy);
  if (sp > K.maxSpeed) {
    float k = fdiv(K.maxSpeed, sp);
    vx = fmul(vx, k); vy = fmul(vy, k);
  }
  if (av > K.maxAngSpeed) av = K.maxAngSpeed;
  else if (av < -K.maxAngSpeed) av = -K.maxAngSpeed;
  if (!(vx == vx) || !(vy == vy)) { vx = 0.f; vy = 0.f; }
  if (!(av == av)) av = 0.f;
  S.vx[i] = vx; S.vy[i] = vy; S.av[i] = av;
  S.ppx[i] = fadd(S.px[i], fmul(K.h, vx));
  S.ppy[i] = fadd(S.py[i], fmul(K.h, vy));
  S.angP[i] = fadd(S.ang[i], fmul(K.h, av));
  S.fx[i] = 0.f; S.fy[i] = 0.f; S.tq[i] = 0.f;
}

// solvePinF, f32solver.mjs:203-256 (solver.wgsl:225-290); grips are pins
// against the world anchor (lbx, lby).
template <class Acc>
__device__ __forceinline__ void solve_pin(const SolverConsts &K, Island &S, int k) {
  int ab = S.ab[k];
  int A = ab & 0xffff, B = (ab >> 16) & 0xffff;
  float sa, ca;
  sincos_r(S.angP[A], &sa, &ca);
  float lax = S.lax[k], lay = S.lay[k];
  float rax = fsub(fmul(lax, ca), fmul(lay, sa));
  float ray = fadd(fmul(lax, sa), fmul(lay, ca));
  float gax = fadd(S.ppx[A], rax), gay = fadd(S.ppy[A], ray);
  float gbx = Acc::lbx(S, k), gby = Acc::lby(S, k);
  float rbx = 0.f, rby = 0.f, wB = 0.f, wIB = 0.f;
  const bool hasB = B != 0xffff;
  if (hasB) {
    float sb, cb;
    sincos_r(S.angP[B], &sb, &cb);
    float lbx = gbx, lby = gby;
    rbx = fsub(fmul(lbx, cb), fmul(lby, sb));
    rby = fadd(fmul(lbx, sb), fmul(lby, cb));
    gbx = fadd(S.ppx[B], rbx); gby = fadd(S.ppy[B], rby);
    wB = S.im[B]; wIB = S.ii[B];
  }
  float Cx = fsub(gax, gbx), Cy = fsub(gay, gby);
  if (!(Cx == Cx) || !(Cy == Cy)) return;
  if (fadd(fmul(Cx, Cx), fmul(Cy, Cy)) < fmul(kSlackPos, kSlackPos)) return;
  float pax = -ray, pay = rax;
  float pbx = -rby, pby = rbx;
  float wA = S.im[A], wIA = S.ii[A];
  float wSum = fadd(wA, wB);
  float k00 = fadd(fadd(wSum, fmul(fmul(wIA, pax), pax)), fmul(fmul(wIB, pbx), pbx));
  float k01 = fadd(fmul(fmul(wIA, pax), pay), fmul(fmul(wIB, pbx), pby));
  float k11 = fadd(fadd(wSum, fmul(fmul(wIA, pay), pay)), fmul(fmul(wIB, pby), pby));
  float det = fsub(fmul(k00, k11), fmul(k01, k01));
  if (fabsf(det) < kEpsDet) return;
  float alphaTilde = fmul(Acc::comp(S, k), K.invH2);
  float lx0 = S.lamX[k], ly0 = S.lamY[k];
  float bx = fadd(Cx, fmul(alphaTilde, lx0));
  float by = fadd(Cy, fmul(alphaTilde, ly0));
  float i00 = fdiv(k11, det), i11 = fdiv(k00, det), i01 = -fdiv(k01, det);
  float dlx = -fadd(fmul(i00, bx), fmul(i01, by));
  float dly = -fadd(fmul(i01, bx), fmul(i11, by));
  if (!(dlx == dlx) || !(dly == dly)) return;
  S.lamX[k] = fadd(lx0, dlx);
  S.lamY[k] = fadd(ly0, dly);
  S.ppx[A] = fadd(S.ppx[A], fmul(wA, dlx));
  S.ppy[A] = fadd(S.ppy[A], fmul(wA, dly));
  S.angP[A] = fadd(S.angP[A], fmul(wIA, fadd(fmul(pax, dlx), fmul(pay, dly))));
  if (hasB) {
    S.ppx[B] = fsub(S.ppx[B], fmul(wB, dlx));
    S.ppy[B] = fsub(S.ppy[B], fmul(wB, dly));
    S.angP[B] = fsub(S.angP[B], fmul(wIB, fadd(fmul(pbx, dlx), fmul(pby, dly))));
  }
}

// solveAngleF, f32solver.mjs:258-301 (solver.wgsl:292-350): muscle
// (compliant) part, then the one-sided joint limit.
template <class Acc>
__device__ __forceinline__ void solve_angle(const SolverConsts &K, Island &S, int k) {
  int ab = S.ab[k];
  int A = ab & 0xffff, B = (ab >> 16) & 0xffff;
  const bool hasB = B != 0xffff;
  float wA = S.ii[A];
  float wB = 0.f;
  float rel = S.angP[A];
  if (hasB) {
    wB = S.ii[B];
    rel = angle_delta(S.angP[B], S.angP[A]);
  }
  float wSum = fadd(wA, wB);
  if (wSum <= 0.f) return;
  float rest = S.rest[k];
  float dev = angle_delta(rel, rest);
  float C = angle_delta(dev, Acc::tgt(S, k));
  if (!(C == C)) return;
  if (fabsf(C) >= kSlackAng) {
    float alphaTilde = fmul(Acc::comp(S, k), K.invH2);
    float l0 = S.lam[k];
    float dl = -fdiv(fadd(C, fmul(alphaTilde, l0)), fadd(wSum, alphaTilde));
    if (!(dl == dl)) return;
    S.lam[k] = fadd(l0, dl);
    if (hasB) {
      S.angP[B] = fadd(S.angP[B], fmul(wB, dl));
      S.angP[A] = fsub(S.angP[A], fmul(wA, dl));
    } else {
      S.angP[A] = fadd(S.angP[A], fmul(wA, dl));
    }
  }
  float rel2 = S.angP[A];
  if (hasB) rel2 = angle_delta(S.angP[B], S.angP[A]);
  float dev2 = angle_delta(rel2, rest);
  float over = 0.f;
  float mx = S.maxA[k], mn = S.minA[k];
  if (dev2 > mx) over = fsub(dev2, mx);
  else if (dev2 < mn) over = fsub(dev2, mn);
  if (fabsf(over) >= kSlackAng) {
    float dl2 = -fdiv(over, wSum);
    if (hasB) {
      S.angP[B] = fadd(S.angP[B], fmul(wB, dl2));
      S.angP[A] = fsub(S.angP[A], fmul(wA, dl2));
    } else {
      S.angP[A] = fadd(S.angP[A], fmul(wA, dl2));
    }
  }
}

// One collision pass of the island: solveCollisionsF 'seq',
// f32solver.mjs:317-344 (solver.wgsl:373-402) -- per body, its points in
// order, each correction cumulative.  Evaluated as
//   1. sin/cos of angP per body (angP does not change in the pass),
//   2. every point at its body's pose at the start of the pass, plus the
//      bounding box of those positions, and the culled rect list,
//   3. per body, the points in order: a point's evaluation from step 2 is
//      the sequential one as long as no earlier point of that body moved
//      it; after the first correction the remaining points of that body are
//      re-evaluated at the moved pose, exactly as the sequential loop does.
// The collision pass with the culled list taken from the box of the bodies'
// centres widened by reach (>= every collision point's distance from its
// body's centre, plus 1 px for rounding): the rects within cull_d of that
// box, in ascending order.  The box holds every point the pass evaluates, so
// the list keeps every rect within cull_d of them and the fold over it is
// exact by the argument above kMaxCulled.  A body with no listed rect within
// reach + cull_d of its centre has no point that any rect can correct: its
// sin/cos, point positions and SDF evaluations are skipped (bc[j] = 2, an
// impossible cosine, marks it) -- its points are unflagged, as the full
// evaluation would leave them.  With an empty list the pass changes nothing
// and ends at once.  Returns false, having changed nothing, when the box is
// not finite or reaches 1e6 px (where 1 px no longer covers f32 rounding) or
// the list would exceed kMaxCulled; the caller then runs the pass below.
template <int G>
__device__ __forceinline__ bool collide_bodies(Island &S, const float4 *__restrict__ rects, int nR, float cull_d,
                                               const Lanes<G> &L, float reach) {
  float lx = __int_as_float(0x7f800000), ly = lx, hx = -lx, hy = -lx;
  for (int j = L.lane; j < S.nb; j += G) {
    lx = fminf(lx, S.ppx[j]); hx = fmaxf(hx, S.ppx[j]);
    ly = fminf(ly, S.ppy[j]); hy = fmaxf(hy, S.ppy[j]);
  }
  lx = L.min(lx); ly = L.min(ly);
  hx = L.max(hx); hy = L.max(hy);
  const float e = reach + cull_d;
  const float x0 = lx - e, x1 = hx + e, y0 = ly - e, y1 = hy + e;
  if (!(x0 <= x1 && y0 <= y1 && fmaxf(fmaxf(fabsf(x0), fabsf(x1)), fmaxf(fabsf(y0), fabsf(y1))) < 1e6f))
    return false;
  int ncull = 0;
  for (int base = 0; base < nR; base += G) {
    const int i = base + L.lane;
    bool keep = false;
    if (i < nR) {
      const float4 r = __ldg(rects + i);
      keep = !(r.z < x0 || r.x > x1 || r.w < y0 || r.y > y1);
    }
    const unsigned m = L.ballot(keep);
    const int at = ncull + __popc(m & ((1u << L.lane) - 1u));
    if (keep && at < kMaxCulled) S.cull[at] = static_cast<short>(i);
    ncull += __popc(m);
    if (ncull > kMaxCulled) {
      L.sync();
      return false;
    }
  }
  if (ncull == 0) return true;
  L.sync();
  for (int j = L.lane; j < S.nb; j += G) {
    const float cx = S.ppx[j], cy = S.ppy[j];
    bool near = false;
    for (int q = 0; q < ncull && !near; q++) {
      const float4 r = __ldg(rects + S.cull[q]);
      near = !(r.z < cx - e || r.x > cx + e || r.w < cy - e || r.y > cy + e);
    }
    if (near) {
      float sn, cs;
      sincos_r(S.angP[j], &sn, &cs);
      S.bs[j] = sn;
      S.bc[j] = cs;
    } else {
      S.bc[j] = 2.f;
    }
  }
  L.sync();
  for (int p = L.lane; p < S.np; p += G) {
    const int j = S.pbody[p];
    const float ca = S.bc[j];
    int flag = 0;
    float cx = 0.f, cy = 0.f;
    if (ca != 2.f && S.im[j] != 0.f) {
      const float sa = S.bs[j], ox = S.plx[p], oy = S.ply[p];
      const float wx = fadd(S.ppx[j], fsub(fmul(ox, ca), fmul(oy, sa)));
      const float wy = fadd(S.ppy[j], fadd(fmul(ox, sa), fmul(oy, ca)));
      float d, nx, ny;
      if (sdf(rects, S.cull, ncull, wx, wy, &d, &nx, &ny)) {
        const float pen = fsub(S.pr[p], d);
        if (pen > kSlackPos) {
          flag = 1;
          cx = fmul(nx, pen);
          cy = fmul(ny, pen);
        }
      }
    }
    S.pflag[p] = flag;
    S.pdx[p] = cx;
    S.pdy[p] = cy;
  }
  L.sync();
  const float sx0 = lx - reach - kCullSlack, sx1 = hx + reach + kCullSlack;
  const float sy0 = ly - reach - kCullSlack, sy1 = hy + reach + kCullSlack;
  for (int j = L.lane; j < S.nb; j += G) {
    if (S.im[j] == 0.f || S.bc[j] == 2.f) continue;
    const int o = S.boff[j], cnt = S.bcnt[j];
    float px = S.ppx[j], py = S.ppy[j];
    const float ca = S.bc[j], sa = S.bs[j];
    bool moved = false;
    for (int q = 0; q < cnt; q++) {
      const int p = o + q;
      if (!moved) {
        if (S.pflag[p]) {
          px = fadd(px, S.pdx[p]);
          py = fadd(py, S.pdy[p]);
          moved = true;
        }
        continue;
      }
      const float ox = S.plx[p], oy = S.ply[p];
      const float wx = fadd(px, fsub(fmul(ox, ca), fmul(oy, sa)));
      const float wy = fadd(py, fadd(fmul(ox, sa), fmul(oy, ca)));
      const bool in_box = wx >= sx0 && wx <= sx1 && wy >= sy0 && wy <= sy1;
      float d, nx, ny;
      if (!sdf(rects, in_box ? S.cull : nullptr, in_box ? ncull : nR, wx, wy, &d, &nx, &ny)) continue;
      const float pen = fsub(S.pr[p], d);
      if (pen <= kSlackPos) continue;
      px = fadd(px, fmul(nx, pen));
      py = fadd(py, fmul(ny, pen));
    }
    S.ppx[j] = px;
    S.ppy[j] = py;
  }
  L.sync();
  return true;
}

// cull_d = D + kCullSlack with D as in the comment above kMaxCulled.  reach
// >= 0 (the batched engine's templates): collide_bodies; reach < 0 (the
// drop-in world, arbitrary collision points): the culled list from the box
// of the evaluated points.
template <int G>
__device__ __forceinline__ void collide_island(Island &S, const float4 *__restrict__ rects, int nR,
                                               float cull_d, const Lanes<G> &L, float reach) {
  if (reach >= 0.f && collide_bodies<G>(S, rects, nR, cull_d, L, reach)) return;
  for (int j = L.lane; j < S.nb; j += G) {
    float s, c;
    sincos_r(S.angP[j], &s, &c);
    S.bs[j] = s;
    S.bc[j] = c;
  }
  L.sync();
  float mnx = __int_as_float(0x7f800000), mny = mnx, mxx = -mnx, mxy = -mnx;
  for (int p = L.lane; p < S.np; p += G) {
    const int j = S.pbody[p];
    const float ca = S.bc[j], sa = S.bs[j], lx = S.plx[p], ly = S.ply[p];
    const float wx = fadd(S.ppx[j], fsub(fmul(lx, ca), fmul(ly, sa)));
    const float wy = fadd(S.ppy[j], fadd(fmul(lx, sa), fmul(ly, ca)));
    S.pdx[p] = wx;  // position for now, correction below
    S.pdy[p] = wy;
    mnx = fminf(mnx, wx); mxx = fmaxf(mxx, wx);
    mny = fminf(mny, wy); mxy = fmaxf(mxy, wy);
  }
  mnx = L.min(mnx); mny = L.min(mny);
  mxx = L.max(mxx); mxy = L.max(mxy);
  // culled list, ascending rect order
  const float bx0 = mnx - cull_d, bx1 = mxx + cull_d, by0 = mny - cull_d, by1 = mxy + cull_d;
  int ncull = 0;
  bool full = !(bx0 <= bx1 && by0 <= by1);  // no finite point: use the full list
  for (int base = 0; base < nR && !full; base += G) {
    const int i = base + L.lane;
    bool keep = false;
    if (i < nR) {
      const float4 r = __ldg(rects + i);
      keep = !(r.z < bx0 || r.x > bx1 || r.w < by0 || r.y > by1);
    }
    const unsigned m = L.ballot(keep);
    const int at = ncull + __popc(m & ((1u << L.lane) - 1u));
    if (keep && at < kMaxCulled) S.cull[at] = static_cast<short>(i);
    ncull += __popc(m);
    if (ncull > kMaxCulled) full = true;
  }
  L.sync();
  const short *list = full ? nullptr : S.cull;
  const int nlist = full ? nR : ncull;
  const float sx0 = mnx - kCullSlack, sx1 = mxx + kCullSlack;
  const float sy0 = mny - kCullSlack, sy1 = mxy + kCullSlack;
  for (int p = L.lane; p < S.np; p += G) {
    const int j = S.pbody[p];
    int flag = 0;
    float cx = 0.f, cy = 0.f;
    if (S.im[j] != 0.f) {
      float d, nx, ny;
      if (sdf(rects, list, nlist, S.pdx[p], S.pdy[p], &d, &nx, &ny)) {
        const float pen = fsub(S.pr[p], d);
        if (pen > kSlackPos) {
          flag = 1;
          cx = fmul(nx, pen);
          cy = fmul(ny, pen);
        }
      }
    }
    S.pflag[p] = flag;
    S.pdx[p] = cx;
    S.pdy[p] = cy;
  }
  L.sync();
  for (int j = L.lane; j < S.nb; j += G) {
    if (S.im[j] == 0.f) continue;
    const int o = S.boff[j], cnt = S.bcnt[j];
    float px = S.ppx[j], py = S.ppy[j];
    const float ca = S.bc[j], sa = S.bs[j];
    bool moved = false;
    for (int q = 0; q < cnt; q++) {
      const int p = o + q;
      if (!moved) {
        if (S.pflag[p]) {
          px = fadd(px, S.pdx[p]);
          py = fadd(py, S.pdy[p]);
          moved = true;
        }
        continue;
      }
      const float lx = S.plx[p], ly = S.ply[p];
      const float wx = fadd(px, fsub(fmul(lx, ca), fmul(ly, sa)));
      const float wy = fadd(py, fadd(fmul(lx, sa), fmul(ly, ca)));
      const bool in_box = wx >= sx0 && wx <= sx1 && wy >= sy0 && wy <= sy1;
      float d, nx, ny;
      if (!sdf(rects, in_box ? list : nullptr, in_box ? nlist : nR, wx, wy, &d, &nx, &ny)) continue;
      const float pen = fsub(S.pr[p], d);
      if (pen <= kSlackPos) continue;
      px = fadd(px, fmul(nx, pen));
      py = fadd(py, fmul(ny, pen));
    }
    S.ppx[j] = px;
    S.ppy[j] = py;
  }
  L.sync();
}

// finalizeF, f32solver.mjs:376-399 (solver.wgsl:405-430)
__device__ __forceinline__ void finalize_body(const SolverConsts &K, Island &S, int i) {
  if (S.im[i] == 0.f && S.ii[i] == 0.f) {
    S.vx[i] = 0.f; S.vy[i] = 0.f; S.av[i] = 0.f;
    return;
  }
  float vx = fmul(fsub(S.ppx[i], S.px[i]), K.invH);
  float vy = fmul(fsub(S.ppy[i], S.py[i]), K.invH);
  float av = fmul(angle_delta(S.angP[i], S.ang[i]), K.invH);
  float sp = length2(vx, vy);
  if (sp > K.maxSpeed) {
    float k = fdiv(K.maxSpeed, sp);
    vx = fmul(vx, k); vy = fmul(vy, k);
  }
  if (av > K.maxAngSpeed) av = K.maxAngSpeed;
  else if (av < -K.maxAngSpeed) av = -K.maxAngSpeed;
  S.vx[i] = vx; S.vy[i] = vy; S.av[i] = av;
  S.px[i] = S.ppx[i]; S.py[i] = S.ppy[i];
  float a = S.angP[i];
  if (a > 50.f || a < -50.f) {
    a = wrap_angle(a);
    S.angP[i] = a;
  }
  S.ang[i] = a;
}

// gripBreakF, f32solver.mjs:402-416 (solver.wgsl:433-442)
template <class Acc>
__device__ __forceinline__ void grip_break(const SolverConsts &K, Island &S, int k) {
  if (Acc::type(S, k) != 2 || Acc::broken(S, k)) return;
  float f = fmul(length2(S.lamX[k], S.lamY[k]), K.invH);
  if (f > Acc::brk(S, k)) {
    Acc::set_broken(S, k);
    S.lamX[k] = 0.f;
    S.lamY[k] = 0.f;
  }
}

// One env step of one island by a group of G lanes (xpbd.js:487-490 with the
// substep of f32solver.mjs:419-428): substeps x (reset lambda, integrate,
// iterations x (constraint levels, collisions), finalize), then grip break.
// U: unroll factor of the substep loop (1: a loop; 2: its body twice per
// trip, remainder handled) -- the same operations in the same order, so the
// results do not depend on it; the batched engine's autotuner picks it.
template <class Acc, int G, int U = 1>
__device__ __forceinline__ void island_step(const SolverConsts &K, Island &S,
                                            const float4 *__restrict__ rects, int nR, float cull_d,
                                            const Lanes<G> &L, float reach) {
#pragma unroll U
  for (int s = 0; s < K.substeps; s++) {
    for (int k = L.lane; k < S.nc; k += G) { S.lamX[k] = 0.f; S.lamY[k] = 0.f; S.lam[k] = 0.f; }
    for (int i = L.lane; i < S.nb; i += G) integrate_body(K, S, i);
    L.sync();
    for (int it = 0; it < K.iterations; it++) {
      for (int l = 0; l < S.nlv; l++) {
        const int beg = S.lvl[l], end = S.lvl[l + 1];
        for (int k = beg + L.lane; k < end; k += G) {
          if (Acc::broken(S, k)) continue;
          if (Acc::type(S, k) == 1) solve_angle<Acc>(K, S, k);
          else solve_pin<Acc>(K, S, k);
        }
        L.sync();
      }
      collide_island<G>(S, rects, nR, cull_d, L, reach);
    }
    for (int i = L.lane; i < S.nb; i += G) finalize_body(K, S, i);
    L.sync();
  }
  for (int k = L.lane; k < S.nc; k += G) grip_break<Acc>(K, S, k);
  L.sync();
}

}  // namespace kr
