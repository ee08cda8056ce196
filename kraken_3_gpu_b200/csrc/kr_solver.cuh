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

// Math.fround(Math.cos(x)), Math.fround(Math.sin(x)) for an f32 argument.
__device__ __forceinline__ void sincos_r(float a, float *s, float *c) {
  double sd, cd;
  sincos(static_cast<double>(a), &sd, &cd);
  *s = static_cast<float>(sd);
  *c = static_cast<float>(cd);
}

// trunc(x / TAU) exactly, as the f64 quotient of f32solver.mjs:38 gives it.
// For |x| >= TAU both x and q*TAU are multiples of 2^-21, so the remainder
// x - q*TAU is exact in one fma and decides whether the rounded f32 quotient
// crossed an integer; for |x| < TAU the truncated quotient is 0 either way.
__device__ __forceinline__ float trunc_quot_tau(float x) {
  float q = truncf(__fdiv_rn(x, kTau));
  float r = fmaf(-q, kTau, x);
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
// sdfF, f32solver.mjs:139-166 (solver.wgsl:114-147).  The division of the
// outward normal is deferred to the final winner: bnx/bny are overwritten by
// every later winner, so only the last winner's dx/best and dy/best survive.
__device__ __forceinline__ bool sdf(const float4 *__restrict__ rects, int nR, float x, float y,
                                    float *od, float *onx, float *ony) {
  float best = kSdfInf, thr = __int_as_float(0x7f800000);  // best*best of 1e30 is +inf in f32
  float wdx = 0.f, wdy = 0.f, inx = 0.f, iny = 0.f;
  bool inside = false;
  for (int i = 0; i < nR; i++) {
    const float4 r = __ldg(rects + i);
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

// Shared-memory view of one island (one warp).  Constraint slots are in
// schedule order: level by level, each level body-disjoint.
struct Island {
  // bodies (local index)
  float *px, *py, *ppx, *ppy, *vx, *vy, *ang, *angP, *av, *im, *ii, *fx, *fy, *tq;
  // constraint slots
  int *ab;     // a | (b << 16), b == 0xffff for a world anchor
  int *tb;     // type | (broken << 8)
  float *lax, *lay, *lbx, *lby, *comp, *rest, *tgt, *minA, *maxA, *lamX, *lamY, *lam, *brk;
  // collision points, grouped per local body in groupCollPoints order
  float *plx, *ply, *pr;
  int *boff, *bcnt;
  int nb, nc, np, nlv, nrounds;
  const int *lvl;        // level offsets, nlv + 1 (global, read-only)
  const short *clane;    // collision lane table, nrounds x 32 (global, read-only)
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
__device__ __forceinline__ void solve_pin(const SolverConsts &K, Island &S, int k) {
  int ab = S.ab[k];
  int A = ab & 0xffff, B = (ab >> 16) & 0xffff;
  float sa, ca;
  sincos_r(S.angP[A], &sa, &ca);
  float lax = S.lax[k], lay = S.lay[k];
  float rax = fsub(fmul(lax, ca), fmul(lay, sa));
  float ray = fadd(fmul(lax, sa), fmul(lay, ca));
  float gax = fadd(S.ppx[A], rax), gay = fadd(S.ppy[A], ray);
  float gbx = S.lbx[k], gby = S.lby[k];
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
  float alphaTilde = fmul(S.comp[k], K.invH2);
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
  float C = angle_delta(dev, S.tgt[k]);
  if (!(C == C)) return;
  if (fabsf(C) >= kSlackAng) {
    float alphaTilde = fmul(S.comp[k], K.invH2);
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

// solveCollisionsF 'seq' for one body, f32solver.mjs:317-344
// (solver.wgsl:373-402): its points in order, each correction cumulative.
// angP does not change inside the loop, so sin/cos are taken once.
__device__ __forceinline__ void collide_body(Island &S, int j, const float4 *__restrict__ rects,
                                             int nR) {
  if (S.im[j] == 0.f) return;
  int cnt = S.bcnt[j];
  if (cnt == 0) return;
  int o = S.boff[j];
  float sa, ca;
  sincos_r(S.angP[j], &sa, &ca);
  float px = S.ppx[j], py = S.ppy[j];
  for (int q = 0; q < cnt; q++) {
    float lx = S.plx[o + q], ly = S.ply[o + q];
    float wx = fadd(px, fsub(fmul(lx, ca), fmul(ly, sa)));
    float wy = fadd(py, fadd(fmul(lx, sa), fmul(ly, ca)));
    float d, nx, ny;
    if (!sdf(rects, nR, wx, wy, &d, &nx, &ny)) continue;
    float pen = fsub(S.pr[o + q], d);
    if (pen <= kSlackPos) continue;
    px = fadd(px, fmul(nx, pen));
    py = fadd(py, fmul(ny, pen));
  }
  S.ppx[j] = px;
  S.ppy[j] = py;
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
__device__ __forceinline__ void grip_break(const SolverConsts &K, Island &S, int k) {
  int tb = S.tb[k];
  if ((tb & 0xff) != 2 || (tb >> 8) != 0) return;
  float f = fmul(length2(S.lamX[k], S.lamY[k]), K.invH);
  if (f > S.brk[k]) {
    S.tb[k] = tb | (1 << 8);
    S.lamX[k] = 0.f;
    S.lamY[k] = 0.f;
  }
}

// One env step of one island by one warp (xpbd.js:487-490 with the substep
// of f32solver.mjs:419-428): substeps x (reset lambda, integrate,
// iterations x (constraint levels, collisions), finalize), then grip break.
__device__ __forceinline__ void island_step(const SolverConsts &K, Island &S,
                                            const float4 *__restrict__ rects, int nR, int lane) {
  for (int s = 0; s < K.substeps; s++) {
    for (int k = lane; k < S.nc; k += 32) { S.lamX[k] = 0.f; S.lamY[k] = 0.f; S.lam[k] = 0.f; }
    for (int i = lane; i < S.nb; i += 32) integrate_body(K, S, i);
    __syncwarp();
    for (int it = 0; it < K.iterations; it++) {
      for (int l = 0; l < S.nlv; l++) {
        const int beg = S.lvl[l], end = S.lvl[l + 1];
        for (int k = beg + lane; k < end; k += 32) {
          const int tb = S.tb[k];
          if ((tb >> 8) != 0) continue;  // broken
          if ((tb & 0xff) == 1) solve_angle(K, S, k);
          else solve_pin(K, S, k);
        }
        __syncwarp();
      }
      for (int r = 0; r < S.nrounds; r++) {
        const int j = S.clane[r * 32 + lane];
        if (j >= 0) collide_body(S, j, rects, nR);
      }
      __syncwarp();
    }
    for (int i = lane; i < S.nb; i += 32) finalize_body(K, S, i);
    __syncwarp();
  }
  for (int k = lane; k < S.nc; k += 32) grip_break(K, S, k);
  __syncwarp();
}

}  // namespace kr
