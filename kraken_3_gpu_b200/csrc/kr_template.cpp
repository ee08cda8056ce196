// kr_template.cpp -- see kr_template.h.
#include "kr_template.h"

#include <algorithm>
#include <cmath>

namespace kr {

namespace {

// BODY, src/body/kraken.js:22-47
constexpr double kPi = 3.141592653589793;
constexpr double kSegLen = 13.5;
constexpr double kShoulderR = 24;
constexpr double kMantleR = 18;
constexpr double kMantleMass = 20;
constexpr double kMantleIF = 2.5;
constexpr double kSegMassProx = 3.2, kSegMassDist = 1.8;
constexpr double kSegThickProx = 11.9, kSegThickDist = 5.9;
constexpr double kStiffMin = 2000;

struct RawCon {
  int type, a, b;
  double lax, lay, lbx, lby, rest, minA, maxA;
  int motor;     // a * segs + j or -1
  int arm;       // owner arm for grips, else -1
  int color;
};

double rect_inertia(double m, double w, double h) { return m * (w * w + h * h) / 12; }

// Levels balanced for G lanes.  Input: the solve list (type and bodies of
// each entry, in list order) and its as-early-as-possible levels.  Any level
// assignment in which every pair of entries sharing a body keeps its list
// order gives bit-identical results (a level holds body-disjoint entries, so
// their order inside it is free).  This one keeps the number of levels and
// each level's constraint type (so a level's lanes never diverge between
// the pin and the angle solve) and fills levels from the first: each level
// takes the entries that cannot go later, then fills its last pass of G
// lanes with the most urgent of the others whose predecessors are placed.
// Returns false (leaving `out` unset) if the list's levels mix types.
bool balance_levels(const std::vector<int> &ty, const std::vector<int> &ea, const std::vector<int> &eb,
                    const std::vector<int> &asap0, int L, int G, std::vector<int> *out) {
  const int n = (int)ty.size();
  std::vector<int> ltype(L, -1);
  for (int i = 0; i < n; i++) {
    if (ltype[asap0[i]] >= 0 && ltype[asap0[i]] != ty[i]) return false;
    ltype[asap0[i]] = ty[i];
  }
  std::vector<std::vector<int>> pred(n), succ(n);
  std::vector<int> last_of;
  for (int i = 0; i < n; i++) {
    for (int b : {ea[i], eb[i]}) {
      if (b < 0) continue;
      if ((int)last_of.size() <= b) last_of.resize(b + 1, -1);
      if (last_of[b] >= 0) { pred[i].push_back(last_of[b]); succ[last_of[b]].push_back(i); }
      last_of[b] = i;
    }
  }
  std::vector<int> asap(n), alap(n);
  for (int i = 0; i < n; i++) {
    int lo = 0;
    for (int p : pred[i]) lo = std::max(lo, asap[p] + 1);
    while (lo < L && ltype[lo] != ty[i]) lo++;
    if (lo >= L) return false;
    asap[i] = lo;
  }
  for (int i = n - 1; i >= 0; i--) {
    int hi = L - 1;
    for (int j : succ[i]) hi = std::min(hi, alap[j] - 1);
    while (hi >= 0 && ltype[hi] != ty[i]) hi--;
    if (hi < asap[i]) return false;
    alap[i] = hi;
  }
  std::vector<int> lvl(n, -1);
  for (int l = 0; l < L; l++) {
    std::vector<int> mand, rest;
    for (int i = 0; i < n; i++) {
      if (lvl[i] >= 0 || ty[i] != ltype[l] || asap[i] > l) continue;
      bool ready = true;
      for (int p : pred[i]) ready = ready && lvl[p] >= 0 && lvl[p] < l;
      if (!ready) continue;
      (alap[i] == l ? mand : rest).push_back(i);
    }
    std::stable_sort(rest.begin(), rest.end(), [&](int x, int y) { return alap[x] < alap[y]; });
    const int cap = std::max(1, (int)(mand.size() + G - 1) / G) * G;
    for (int i : mand) lvl[i] = l;
    for (size_t k = 0; k < rest.size() && (int)(mand.size() + k) < cap; k++) lvl[rest[k]] = l;
  }
  for (int i = 0; i < n; i++) {
    if (lvl[i] < 0) return false;
    for (int j : succ[i])
      if (lvl[i] >= lvl[j]) return false;
  }
  *out = lvl;
  return true;
}

}  // namespace

bool build_template(int arms, int segs, Template *t, std::string *err) {
  if (arms < 1 || arms > kMaxArms || segs < 1 || segs > kMaxSegs) {
    *err = "body shape " + std::to_string(arms) + "x" + std::to_string(segs) +
           " outside 1.." + std::to_string(kMaxArms) + " arms x 1.." + std::to_string(kMaxSegs) +
           " segments";
    return false;
  }
  *t = Template();
  t->arms = arms;
  t->segs = segs;
  t->reach = kShoulderR + segs * kSegLen;
  const double joint = kPi * 0.42, shoulder = kPi * 0.62;
  std::vector<double> im, ii;
  std::vector<int> pbody;
  std::vector<double> plx, ply, pr;
  std::vector<RawCon> cons;
  auto add_body = [&](double mass, double inertia) {
    im.push_back(mass > 0 ? 1 / mass : 0);
    ii.push_back(inertia > 0 ? 1 / inertia : 0);
    return (int)im.size() - 1;
  };
  auto add_pt = [&](int b, double lx, double ly, double r) {
    pbody.push_back(b); plx.push_back(lx); ply.push_back(ly); pr.push_back(r);
  };
  auto add_con = [&](int type, int a, int b, double lax, double lay, double lbx, double lby) {
    RawCon c{type, a, b, lax, lay, lbx, lby, 0, -INFINITY, INFINITY, -1, -1, -1};
    cons.push_back(c);
    return (int)cons.size() - 1;
  };
  // spawnKraken creation order (kraken.js:64-148)
  const double mantleI = (kMantleMass * kMantleR * kMantleR / 2) * kMantleIF;
  const int mantle = add_body(kMantleMass, mantleI);
  for (int i = 0; i < 8; i++) {
    const double a = ((double)i / 8) * kPi * 2;
    add_pt(mantle, std::cos(a) * kMantleR * 0.7, std::sin(a) * kMantleR * 0.7, kMantleR * 0.45);
  }
  t->arm_tip.resize(arms);
  t->arm_seg0.resize(arms);
  t->arm_segs.resize((size_t)arms * segs);
  std::vector<int> grip_raw(arms);
  for (int a = 0; a < arms; a++) {
    const double relAng = ((double)a / arms) * kPi * 2;
    std::vector<int> sg(segs);
    for (int i = 0; i < segs; i++) {
      const double tt = segs > 1 ? (double)i / (segs - 1) : 0;
      const double mass = kSegMassProx + (kSegMassDist - kSegMassProx) * tt;
      const double thick = kSegThickProx + (kSegThickDist - kSegThickProx) * tt;
      const int b = add_body(mass, rect_inertia(mass, kSegLen, thick));
      const double r = thick * 0.5;
      add_pt(b, -kSegLen * 0.5 + r * 0.4, 0, r);
      add_pt(b, kSegLen * 0.5 - r * 0.4, 0, r);
      sg[i] = b;
      t->arm_segs[(size_t)a * segs + i] = b;
    }
    add_con(0, mantle, sg[0], std::cos(relAng) * kShoulderR, std::sin(relAng) * kShoulderR,
            -kSegLen * 0.5, 0);
    int ms = add_con(1, mantle, sg[0], 0, 0, 0, 0);
    cons[ms].rest = relAng;
    cons[ms].minA = -shoulder;
    cons[ms].maxA = shoulder;
    cons[ms].motor = a * segs;
    for (int i = 0; i + 1 < segs; i++) {
      add_con(0, sg[i], sg[i + 1], kSegLen * 0.5, 0, -kSegLen * 0.5, 0);
      int m = add_con(1, sg[i], sg[i + 1], 0, 0, 0, 0);
      cons[m].rest = 0.28;  // spawnCurl: the spawn pose is the fixpoint
      cons[m].minA = -joint;
      cons[m].maxA = joint;
      cons[m].motor = a * segs + i + 1;
    }
    int g = add_con(2, sg[segs - 1], -1, kSegLen * 0.5, 0, 0, 0);
    cons[g].arm = a;
    grip_raw[a] = g;
    t->arm_tip[a] = sg[segs - 1];
    t->arm_seg0[a] = sg[0];
  }
  const int nb = (int)im.size(), nc = (int)cons.size(), np = (int)pbody.size();
  // colouring in creation order (core.js:51-58 / assignColor) and stable grouping
  std::vector<uint32_t> mask(nb, 0u);
  for (auto &c : cons) {
    uint32_t used = mask[c.a] | (c.b >= 0 ? mask[c.b] : 0u);
    int col = 0;
    while (col < 31 && (used & (1u << col))) col++;
    mask[c.a] |= 1u << col;
    if (c.b >= 0) mask[c.b] |= 1u << col;
    c.color = col;
  }
  std::vector<int> list(nc);
  for (int i = 0; i < nc; i++) list[i] = i;
  std::stable_sort(list.begin(), list.end(),
                   [&](int x, int y) { return cons[x].color < cons[y].color; });
  // levels from the list order
  std::vector<int> last(nb, -1), level(nc);
  int nlv = 0;
  for (int q = 0; q < nc; q++) {
    const RawCon &c = cons[list[q]];
    int L = last[c.a] + 1;
    if (c.b >= 0) L = std::max(L, last[c.b] + 1);
    level[q] = L;
    last[c.a] = L;
    if (c.b >= 0) last[c.b] = L;
    nlv = std::max(nlv, L + 1);
  }
  if (nlv > kMaxTplLevels) {
    *err = "body shape needs " + std::to_string(nlv) + " levels";
    return false;
  }
  t->nb = nb; t->nc = nc; t->np = np;
  t->im.resize(nb); t->ii.resize(nb);
  for (int i = 0; i < nb; i++) { t->im[i] = (float)im[i]; t->ii[i] = (float)ii[i]; }
  // the list's types and bodies, for the balanced schedules
  std::vector<int> lty(nc), la(nc), lb(nc);
  for (int q = 0; q < nc; q++) {
    const RawCon &c = cons[list[q]];
    lty[q] = c.type == 1 ? 1 : 0;
    la[q] = c.a;
    lb[q] = c.b;
  }
  for (int v = 0; v < kSchedules; v++) {
    const int G = v == 0 ? 32 : v == 1 ? 16 : 8;
    std::vector<int> lv = level, bal;
    if (balance_levels(lty, la, lb, level, nlv, G, &bal)) lv = bal;
    Schedule &S = t->sched[v];
    S.nlv = nlv;
    std::vector<int> cnt(nlv + 1, 0);
    for (int q = 0; q < nc; q++) cnt[lv[q] + 1]++;
    for (int L = 0; L < nlv; L++) cnt[L + 1] += cnt[L];
    std::vector<int> order(nc), cur(cnt.begin(), cnt.end() - 1);
    for (int q = 0; q < nc; q++) order[cur[lv[q]]++] = list[q];
    S.lvl = cnt;
    std::vector<int> slot_of(nc);
    for (int s = 0; s < nc; s++) {
      const RawCon &c = cons[order[s]];
      slot_of[order[s]] = s;
      const uint32_t b = c.b >= 0 ? (uint32_t)c.b : 0xffffu;
      S.ab.push_back((int)((uint32_t)c.a | (b << 16)));
      S.type.push_back(c.type);
      S.lax.push_back((float)c.lax); S.lay.push_back((float)c.lay);
      S.lbx.push_back((float)c.lbx); S.lby.push_back((float)c.lby);
      S.rest.push_back((float)c.rest);
      S.minA.push_back((float)c.minA); S.maxA.push_back((float)c.maxA);
      S.motor.push_back(c.motor);
    }
    S.arm_grip.resize(arms);
    for (int a = 0; a < arms; a++) S.arm_grip[a] = slot_of[grip_raw[a]];
  }
  const Schedule &S0 = t->sched[0];
  t->nlv = nlv;
  t->lvl = S0.lvl;
  t->ab = S0.ab; t->type = S0.type; t->motor = S0.motor;
  t->lax = S0.lax; t->lay = S0.lay; t->lbx = S0.lbx; t->lby = S0.lby;
  t->rest = S0.rest; t->minA = S0.minA; t->maxA = S0.maxA;
  t->arm_grip = S0.arm_grip;
  // points grouped per body, creation order within a body (groupCollPoints)
  t->boff.assign(nb, 0);
  t->bcnt.assign(nb, 0);
  for (int p = 0; p < np; p++) t->bcnt[pbody[p]]++;
  int acc = 0;
  for (int b = 0; b < nb; b++) { t->boff[b] = acc; acc += t->bcnt[b]; }
  t->plx.assign(np, 0.f); t->ply.assign(np, 0.f); t->pr.assign(np, 0.f); t->pbody.assign(np, 0);
  std::vector<int> pc = t->boff;
  for (int p = 0; p < np; p++) {
    const int q = pc[pbody[p]]++;
    t->plx[q] = (float)plx[p]; t->ply[q] = (float)ply[p]; t->pr[q] = (float)pr[p];
    t->pbody[q] = pbody[p];
    t->r_max = std::max(t->r_max, (float)pr[p]);
    const double off = std::sqrt((double)t->plx[q] * t->plx[q] + (double)t->ply[q] * t->ply[q]);
    t->off_max = std::max(t->off_max, (float)off);
  }
  return true;
}

void spawn_pose(const Template &t, double x, double y, double angle, double curl, double *px,
                double *py, double *ang) {
  px[0] = x; py[0] = y; ang[0] = angle;
  for (int a = 0; a < t.arms; a++) {
    const double relAng = ((double)a / t.arms) * kPi * 2;
    const double th0 = angle + relAng;
    double jx = x + std::cos(th0) * kShoulderR;
    double jy = y + std::sin(th0) * kShoulderR;
    double th = th0;
    for (int i = 0; i < t.segs; i++) {
      const double ux = std::cos(th), uy = std::sin(th);
      const double cx = jx + ux * kSegLen * 0.5;
      const double cy = jy + uy * kSegLen * 0.5;
      const int b = t.arm_segs[(size_t)a * t.segs + i];
      px[b] = cx; py[b] = cy; ang[b] = th;
      jx = cx + ux * kSegLen * 0.5;
      jy = cy + uy * kSegLen * 0.5;
      th += curl;
    }
  }
}

}  // namespace kr
