// kr_world.cu -- the gpuworld.js drop-in: handle, schedule and the plain
// per-step kernel (one launch per env step, one warp per creature).
//
// Device buffers hold the reference's own AoS blocks (48 B bodies, 80 B
// constraints, 16 B forces / collision points), so upload and download are
// single copies and mirrorInto/packControls keep their exact field offsets.
// The kernel stages each creature into shared memory as SoA for the launch.
//
// Schedule.  The reference runs one dispatch per colour class
// (gpuworld.js:353-366); a colour class is body-disjoint, so the classes in
// order are one valid sequential order of the solve list.  Here every
// connected component of the constraint graph (a creature) gets its own
// schedule: each constraint is placed on the first level after every earlier
// constraint (in solve-list order) that shares one of its bodies.  Levels are
// body-disjoint, and any order that keeps every pair of constraints sharing a
// body in list order gives bit-identical results (the harness check
// color-order-free, harness.js:1172-1193, pins this property for the
// reference), so the warp's level sweep reproduces the list order exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/kraken_b200.h"
#include "kr_solver.cuh"

namespace {

thread_local std::string g_last_error;

constexpr int kWarpsPerBlock = 4;

// Per-island record, one int array of kIslandInts per island.
enum { I_BODY_OFF = 0, I_NB, I_CON_OFF, I_NC, I_PT_OFF, I_NP, I_LVL_OFF, I_NLV, kIslandInts };

struct DeviceTables {
  const int *isl;          // nI x kIslandInts
  const int *bodies;       // global body id per island body
  const int *cons;         // global constraint index per schedule slot
  const int *ab;           // local a | local b << 16 per schedule slot
  const int *pts;          // global collision point index, local-body grouped
  const int2 *bpt;         // per island body: (offset within island points, count)
  const int *lvl;          // level offsets per island (nlv + 1 each)
};

struct StepArgs {
  kr::SolverConsts K;
  float *bodies;           // nB x 12
  uint32_t *cons;          // nC x 20
  float *forces;           // nB x 4
  const uint4 *coll;       // nP x 4 words
  const float4 *rects;     // nR x (x, y, x+w, y+h)
  int nR;
  float cull_d;            // rect culling distance of a collision pass
  float reach;             // bound on a collision point's distance from its body (+1 px), < 0: none
  int nI;
  int maxB, maxC, maxP;    // smem carve sizes (per warp)
  DeviceTables T;
};

__host__ __device__ inline int warp_smem_words(int mb, int mc, int mp) {
  return 18 * mb + 15 * mc + 7 * mp + kr::kMaxCulled / 2;
}

// Writable views of the per-slot statics while they are staged; the solver
// reads them through the const pointers of kr::Island.
struct StageView {
  int *ab, *boff, *bcnt, *pbody;
  float *lax, *lay, *rest, *minA, *maxA, *plx, *ply, *pr;
};

__device__ inline void carve(kr::Island &S, StageView &V, float *base, int mb, int mc, int mp) {
  float *p = base;
  S.px = p; p += mb; S.py = p; p += mb; S.ppx = p; p += mb; S.ppy = p; p += mb;
  S.vx = p; p += mb; S.vy = p; p += mb; S.ang = p; p += mb; S.angP = p; p += mb;
  S.av = p; p += mb; S.im = p; p += mb; S.ii = p; p += mb;
  S.fx = p; p += mb; S.fy = p; p += mb; S.tq = p; p += mb;
  S.bs = p; p += mb; S.bc = p; p += mb;
  V.boff = reinterpret_cast<int *>(p); p += mb;
  V.bcnt = reinterpret_cast<int *>(p); p += mb;
  V.ab = reinterpret_cast<int *>(p); p += mc;
  S.tb = reinterpret_cast<int *>(p); p += mc;
  V.lax = p; p += mc; V.lay = p; p += mc; S.lbx = p; p += mc; S.lby = p; p += mc;
  S.comp = p; p += mc; V.rest = p; p += mc; S.tgt = p; p += mc; V.minA = p; p += mc;
  V.maxA = p; p += mc; S.lamX = p; p += mc; S.lamY = p; p += mc; S.lam = p; p += mc;
  S.brk = p; p += mc;
  V.plx = p; p += mp; V.ply = p; p += mp; V.pr = p; p += mp;
  S.pdx = p; p += mp; S.pdy = p; p += mp;
  V.pbody = reinterpret_cast<int *>(p); p += mp;
  S.pflag = reinterpret_cast<int *>(p); p += mp;
  S.cull = reinterpret_cast<short *>(p);
  S.ab = V.ab; S.boff = V.boff; S.bcnt = V.bcnt; S.pbody = V.pbody;
  S.lax = V.lax; S.lay = V.lay; S.rest = V.rest; S.minA = V.minA; S.maxA = V.maxA;
  S.plx = V.plx; S.ply = V.ply; S.pr = V.pr;
}

// One launch of the plain step for the island of this warp (shared by the
// plain kernel and its allocation-free variant).
__device__ __forceinline__ void plain_step_body(const StepArgs &A) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int island = blockIdx.x * kWarpsPerBlock + warp;
  if (island >= A.nI) return;
  kr::Island S;
  StageView V;
  carve(S, V, smem + warp * warp_smem_words(A.maxB, A.maxC, A.maxP), A.maxB, A.maxC, A.maxP);
  const int *rec = A.T.isl + island * kIslandInts;
  const int bo = rec[I_BODY_OFF], co = rec[I_CON_OFF], po = rec[I_PT_OFF];
  S.nb = rec[I_NB]; S.nc = rec[I_NC]; S.np = rec[I_NP];
  S.nlv = rec[I_NLV];
  S.lvl = A.T.lvl + rec[I_LVL_OFF];

  // stage bodies (48 B AoS -> SoA) and forces
  for (int i = lane; i < S.nb; i += 32) {
    const int g = A.T.bodies[bo + i];
    const float4 *b4 = reinterpret_cast<const float4 *>(A.bodies + 12 * (size_t)g);
    const float4 q0 = b4[0], q1 = b4[1], q2 = b4[2];
    S.px[i] = q0.x; S.py[i] = q0.y; S.ppx[i] = q0.z; S.ppy[i] = q0.w;
    S.vx[i] = q1.x; S.vy[i] = q1.y; S.ang[i] = q1.z; S.angP[i] = q1.w;
    S.av[i] = q2.x; S.im[i] = q2.y; S.ii[i] = q2.z;
    const float4 f = reinterpret_cast<const float4 *>(A.forces)[g];
    S.fx[i] = f.x; S.fy[i] = f.y; S.tq[i] = f.z;
    const int2 bp = A.T.bpt[bo + i];
    V.boff[i] = bp.x; V.bcnt[i] = bp.y;
    for (int q = 0; q < bp.y; q++) V.pbody[bp.x + q] = i;
  }
  // stage constraints (80 B AoS -> SoA, schedule order)
  for (int k = lane; k < S.nc; k += 32) {
    const int g = A.T.cons[co + k];
    const uint4 *c4 = reinterpret_cast<const uint4 *>(A.cons + 20 * (size_t)g);
    const uint4 w0 = c4[0], w1 = c4[1], w2 = c4[2], w3 = c4[3], w4 = c4[4];
    V.ab[k] = A.T.ab[co + k];
    S.tb[k] = static_cast<int>(w0.z & 0xffu) | ((w4.y != 0u ? 1 : 0) << 8);
    V.lax[k] = __uint_as_float(w1.x); V.lay[k] = __uint_as_float(w1.y);
    S.lbx[k] = __uint_as_float(w1.z); S.lby[k] = __uint_as_float(w1.w);
    S.comp[k] = __uint_as_float(w2.x); V.rest[k] = __uint_as_float(w2.y);
    S.tgt[k] = __uint_as_float(w2.z); V.minA[k] = __uint_as_float(w2.w);
    V.maxA[k] = __uint_as_float(w3.x); S.lamX[k] = __uint_as_float(w3.y);
    S.lamY[k] = __uint_as_float(w3.z); S.lam[k] = __uint_as_float(w3.w);
    S.brk[k] = __uint_as_float(w4.x);
  }
  // stage collision points
  for (int p = lane; p < S.np; p += 32) {
    const uint4 cp = A.coll[A.T.pts[po + p]];
    V.plx[p] = __uint_as_float(cp.y); V.ply[p] = __uint_as_float(cp.z);
    V.pr[p] = __uint_as_float(cp.w);
  }
  __syncwarp();

  kr::island_step<kr::SlotAccess, 32>(A.K, S, A.rects, A.nR, A.cull_d, kr::Lanes<32>(lane), A.reach);

  // write back bodies, consumed forces and constraint multipliers / flags
  for (int i = lane; i < S.nb; i += 32) {
    const int g = A.T.bodies[bo + i];
    float4 *b4 = reinterpret_cast<float4 *>(A.bodies + 12 * (size_t)g);
    const float pad = A.bodies[12 * (size_t)g + 11];
    b4[0] = make_float4(S.px[i], S.py[i], S.ppx[i], S.ppy[i]);
    b4[1] = make_float4(S.vx[i], S.vy[i], S.ang[i], S.angP[i]);
    b4[2] = make_float4(S.av[i], S.im[i], S.ii[i], pad);
    if (!(S.im[i] == 0.f && S.ii[i] == 0.f)) {
      float *f = A.forces + 4 * (size_t)g;
      f[0] = 0.f; f[1] = 0.f; f[2] = 0.f;  // consumed, adhesion kept (solver.wgsl:204)
    }
  }
  for (int k = lane; k < S.nc; k += 32) {
    const int g = A.T.cons[co + k];
    uint32_t *c = A.cons + 20 * (size_t)g;
    c[13] = __float_as_uint(S.lamX[k]);
    c[14] = __float_as_uint(S.lamY[k]);
    c[15] = __float_as_uint(S.lam[k]);
    c[17] = (S.tb[k] >> 8) != 0 ? 1u : 0u;
  }
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock) plain_step_kernel(StepArgs A) {
  plain_step_body(A);
}

template <typename T>
cudaError_t dev_upload(T **dptr, size_t *cap, const std::vector<T> &v) {
  size_t n = std::max<size_t>(v.size(), 1);
  if (*dptr == nullptr || *cap < n) {
    if (*dptr) cudaFree(*dptr);
    *dptr = nullptr;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(dptr), n * sizeof(T));
    if (e != cudaSuccess) return e;
    *cap = n;
  }
  if (v.empty()) return cudaSuccess;
  return cudaMemcpy(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

struct kr_world {
  kr_solver_params p{};
  kr::SolverConsts K{};
  uint32_t nB = 0, nC = 0, nP = 0, nR = 0;
  float *d_bodies = nullptr;
  uint32_t *d_cons = nullptr;
  uint32_t *d_stage = nullptr;          // staging copy of a control upload
  size_t smem_bytes = 0;
  float *d_forces = nullptr;
  float4 *d_rects = nullptr;
  uint4 *d_coll = nullptr;
  std::vector<uint32_t> h_coll_range;   // 2 x nB
  // island tables
  int *d_isl = nullptr, *d_ibodies = nullptr, *d_icons = nullptr, *d_iab = nullptr,
      *d_ipts = nullptr, *d_lvl = nullptr;
  int2 *d_bpt = nullptr;
  size_t c_isl = 0, c_ibodies = 0, c_icons = 0, c_iab = 0, c_ipts = 0, c_lvl = 0, c_bpt = 0;
  float max_half_thick = 0.f;  // largest min(w, h) / 2 of the map's rects
  float cull_d = 0.f;
  float reach = -1.f;          // largest collision-point offset + 1 px (kr_solver.cuh collide_bodies)
  int nI = 0, maxB = 1, maxC = 1, maxP = 1, maxLv = 0;
  bool uploaded = false;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;

  int fail(int code, const std::string &msg) {
    err = msg;
    return code;
  }
  int cuda_fail(cudaError_t e, const char *what) {
    err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return KR_ERR_CUDA;
  }
};

extern "C" int kr_device_count(void) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    g_last_error = std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e);
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" const char *kr_last_error(const kr_world *w) {
  if (w) return w->err.c_str();
  return g_last_error.c_str();
}

extern "C" int kr_create(const kr_solver_params *params, uint32_t n_bodies, uint32_t n_constraints,
                         const float *rects, uint32_t n_rects, const uint32_t *coll_pts,
                         uint32_t n_coll_pts, const uint32_t *coll_range, kr_world **out) {
  if (!out || !params) {
    g_last_error = "kr_create: null argument";
    return KR_ERR_INVALID;
  }
  *out = nullptr;
  const kr_solver_params &p = *params;
  // sanity guards of writeStatic (gpuworld.js:224-229), same bounds
  if (!(p.iterations >= 1 && p.iterations <= 64)) {
    g_last_error = "iterations implausible: " + std::to_string(p.iterations);
    return KR_ERR_INVALID;
  }
  if (!(n_rects >= 1 && n_rects <= 100000)) {
    g_last_error = "nRects implausible: " + std::to_string(n_rects);
    return KR_ERR_INVALID;
  }
  if (!(n_bodies >= 1 && n_bodies <= 4000000)) {
    g_last_error = "nBodies implausible: " + std::to_string(n_bodies);
    return KR_ERR_INVALID;
  }
  const float hf = static_cast<float>(p.h);
  if (!(hf > 0.f && hf < 1.f)) {
    g_last_error = "h implausible: " + std::to_string(p.h);
    return KR_ERR_INVALID;
  }
  if (p.substeps < 1 || p.substeps > 64) {
    g_last_error = "substeps implausible: " + std::to_string(p.substeps);
    return KR_ERR_INVALID;
  }
  if ((n_coll_pts > 0 && (!coll_pts || !coll_range)) || !rects) {
    g_last_error = "kr_create: missing rects or collision points";
    return KR_ERR_INVALID;
  }
  // collRange must cover the points exactly (gpuworld.js:193-199)
  uint64_t acc = 0;
  if (coll_range) {
    for (uint32_t b = 0; b < n_bodies; b++) {
      if (coll_range[b] != acc) {
        g_last_error = "collRange offsets are not contiguous at body " + std::to_string(b);
        return KR_ERR_INVALID;
      }
      acc += coll_range[n_bodies + b];
    }
    for (uint32_t i = 0; i < n_coll_pts; i++) {
      if (coll_pts[4 * i] >= n_bodies) {
        g_last_error = "collPt " + std::to_string(i) + " refers to body " +
                       std::to_string(coll_pts[4 * i]) + " of " + std::to_string(n_bodies);
        return KR_ERR_INDEX;
      }
    }
  }
  if (acc != n_coll_pts) {
    g_last_error = "collRange covers " + std::to_string(acc) + " of " +
                   std::to_string(n_coll_pts) + " points";
    return KR_ERR_INVALID;
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    cudaGetLastError();
    g_last_error = "no CUDA device available";
    return KR_ERR_NODEVICE;
  }

  kr_world *w = new kr_world();
  w->p = p;
  w->nB = n_bodies; w->nC = n_constraints; w->nP = n_coll_pts; w->nR = n_rects;
  // f32 constants: writeStatic F[0], F[10], F[11] and f32solver.mjs:79-85
  kr::SolverConsts &K = w->K;
  K.h = hf;
  K.invH = static_cast<float>(1.0 / p.h);
  K.invH2 = static_cast<float>(1.0 / (p.h * p.h));
  const float nl = -static_cast<float>(p.lin_drag), na = -static_cast<float>(p.ang_drag);
  K.linDamp = static_cast<float>(std::exp(static_cast<double>(nl * hf)));
  K.angDamp = static_cast<float>(std::exp(static_cast<double>(na * hf)));
  K.maxSpeed = static_cast<float>(p.max_speed);
  K.maxAngSpeed = static_cast<float>(p.max_ang_speed);
  K.substeps = p.substeps;
  K.iterations = p.iterations;

  cudaError_t e;
  auto cleanup_fail = [&](cudaError_t ce, const char *what) {
    g_last_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(ce);
    kr_destroy(w);
    return KR_ERR_CUDA;
  };
  if ((e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return cleanup_fail(e, "cudaStreamCreate");
  w->own_stream = true;
  if ((e = cudaMalloc(&w->d_bodies, sizeof(float) * 12 * n_bodies)) != cudaSuccess)
    return cleanup_fail(e, "cudaMalloc(bodies)");
  if ((e = cudaMalloc(&w->d_cons, sizeof(uint32_t) * 20 * std::max<uint32_t>(n_constraints, 1))) !=
      cudaSuccess)
    return cleanup_fail(e, "cudaMalloc(cons)");
  if ((e = cudaMalloc(&w->d_stage, sizeof(uint32_t) * 20 * std::max<uint32_t>(n_constraints, 1))) !=
      cudaSuccess)
    return cleanup_fail(e, "cudaMalloc(control staging)");
  if ((e = cudaMalloc(&w->d_forces, sizeof(float) * 4 * n_bodies)) != cudaSuccess)
    return cleanup_fail(e, "cudaMalloc(forces)");
  if ((e = cudaMemset(w->d_forces, 0, sizeof(float) * 4 * n_bodies)) != cudaSuccess)
    return cleanup_fail(e, "cudaMemset(forces)");
  std::vector<float4> r4(n_rects);
  double half_thick = 0.0, r_max = 0.0;
  for (uint32_t i = 0; i < n_rects; i++) {
    const float x = rects[4 * i], y = rects[4 * i + 1], rw = rects[4 * i + 2], rh = rects[4 * i + 3];
    r4[i] = make_float4(x, y, x + rw, y + rh);  // f32 sums, as solver.wgsl:120-121
    const double ht = 0.5 * std::min(std::fabs((double)rw), std::fabs((double)rh));
    if (std::isfinite(ht)) half_thick = std::max(half_thick, ht);
    else half_thick = HUGE_VAL;
  }
  double off_max = 0.0;
  for (uint32_t i = 0; i < n_coll_pts; i++) {
    float r, lx, ly;
    std::memcpy(&lx, &coll_pts[4 * i + 1], sizeof(float));
    std::memcpy(&ly, &coll_pts[4 * i + 2], sizeof(float));
    std::memcpy(&r, &coll_pts[4 * i + 3], sizeof(float));
    if (std::isfinite(r)) r_max = std::max(r_max, std::fabs((double)r));
    else r_max = HUGE_VAL;
    const double off = std::sqrt((double)lx * lx + (double)ly * ly);
    off_max = std::isfinite(off) ? std::max(off_max, off) : HUGE_VAL;
  }
  // every collision point lies within off_max of its body's centre: the
  // collision pass may skip bodies with no rect nearby (collide_bodies)
  w->reach = off_max < 1e5 ? (float)off_max + 1.f : -1.f;
  // D = max(radius, half thickness) + 2, plus the slack of the culling box;
  // the f32 rounding of the box test is covered by the +1
  const double cull = std::max(r_max, half_thick) + 2.0 + kr::kCullSlack + 1.0;
  w->cull_d = std::isfinite(cull) && cull < 1e30 ? (float)cull : 1e30f;
  w->max_half_thick = (float)std::min(half_thick, 1e30);
  if ((e = cudaMalloc(&w->d_rects, sizeof(float4) * n_rects)) != cudaSuccess)
    return cleanup_fail(e, "cudaMalloc(rects)");
  if ((e = cudaMemcpy(w->d_rects, r4.data(), sizeof(float4) * n_rects, cudaMemcpyHostToDevice)) !=
      cudaSuccess)
    return cleanup_fail(e, "cudaMemcpy(rects)");
  if ((e = cudaMalloc(&w->d_coll, sizeof(uint4) * std::max<uint32_t>(n_coll_pts, 1))) != cudaSuccess)
    return cleanup_fail(e, "cudaMalloc(collPts)");
  if (n_coll_pts &&
      (e = cudaMemcpy(w->d_coll, coll_pts, sizeof(uint4) * n_coll_pts, cudaMemcpyHostToDevice)) !=
          cudaSuccess)
    return cleanup_fail(e, "cudaMemcpy(collPts)");
  w->h_coll_range.assign(2 * (size_t)n_bodies, 0u);
  if (coll_range) std::memcpy(w->h_coll_range.data(), coll_range, sizeof(uint32_t) * 2 * n_bodies);
  *out = w;
  return KR_OK;
}

namespace {

// Connected components, per-component levels and lane tables (see the file
// comment).  Returns KR_OK or an error code with w->err set.
int build_schedule(kr_world *w, const float *bodies, const uint32_t *cons) {
  const uint32_t nB = w->nB, nC = w->nC;
  std::vector<int> parent(nB);
  std::iota(parent.begin(), parent.end(), 0);
  auto find = [&](int x) {
    while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; }
    return x;
  };
  for (uint32_t k = 0; k < nC; k++) {
    const uint32_t a = cons[20 * k], b = cons[20 * k + 1];
    if (a >= nB || (b != 0xffffffffu && b >= nB)) {
      return w->fail(KR_ERR_INDEX, "Constraint " + std::to_string(k) + ": body index " +
                                       std::to_string(a) + "/" +
                                       (b == 0xffffffffu ? std::string("-1") : std::to_string(b)) +
                                       " outside of " + std::to_string(nB) +
                                       " (an out-of-bounds read in the kernel)");
    }
    if (b != 0xffffffffu) {
      int ra = find((int)a), rb = find((int)b);
      if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
    }
  }
  // islands in order of their smallest body
  std::vector<int> island_of(nB), local(nB);
  std::vector<std::vector<int>> ib;  // bodies per island
  std::vector<int> root_island(nB, -1);
  for (uint32_t g = 0; g < nB; g++) {
    int r = find((int)g);
    if (root_island[r] < 0) { root_island[r] = (int)ib.size(); ib.emplace_back(); }
    int I = root_island[r];
    island_of[g] = I;
    local[g] = (int)ib[I].size();
    ib[I].push_back((int)g);
  }
  const int nI = (int)ib.size();
  std::vector<std::vector<int>> ic(nI);  // constraints per island, list order
  for (uint32_t k = 0; k < nC; k++) ic[island_of[cons[20 * k]]].push_back((int)k);

  std::vector<int> isl(nI * (size_t)kIslandInts), h_bodies, h_cons, h_ab, h_pts, h_lvl;
  std::vector<int2> h_bpt;
  h_bodies.reserve(nB); h_cons.reserve(nC); h_ab.reserve(nC);
  int maxB = 1, maxC = 1, maxP = 1, maxLv = 0;
  std::vector<int> last_level, level, order, cnt_per_level;
  for (int I = 0; I < nI; I++) {
    const auto &bl = ib[I];
    const auto &cl = ic[I];
    const int nb = (int)bl.size(), nc = (int)cl.size();
    if (nb > KR_MAX_ISLAND_BODIES || nc > KR_MAX_ISLAND_CONSTRAINTS)
      return w->fail(KR_ERR_CAPACITY, "connected component " + std::to_string(I) + " has " +
                                          std::to_string(nb) + " bodies and " +
                                          std::to_string(nc) + " constraints; the kernel holds " +
                                          std::to_string(KR_MAX_ISLAND_BODIES) + " / " +
                                          std::to_string(KR_MAX_ISLAND_CONSTRAINTS));
    int *rec = &isl[I * (size_t)kIslandInts];
    rec[I_BODY_OFF] = (int)h_bodies.size();
    rec[I_NB] = nb;
    for (int g : bl) h_bodies.push_back(g);
    // levels: first level after every earlier constraint sharing a body
    last_level.assign(nb, -1);
    level.resize(nc);
    int nlv = 0;
    for (int q = 0; q < nc; q++) {
      const uint32_t *c = cons + 20 * (size_t)cl[q];
      const int a = local[c[0]];
      const int b = c[1] == 0xffffffffu ? -1 : local[c[1]];
      int L = last_level[a] + 1;
      if (b >= 0) L = std::max(L, last_level[b] + 1);
      level[q] = L;
      last_level[a] = L;
      if (b >= 0) last_level[b] = L;
      nlv = std::max(nlv, L + 1);
    }
    if (nlv > KR_MAX_LEVELS)
      return w->fail(KR_ERR_CAPACITY, "connected component " + std::to_string(I) + " needs " +
                                          std::to_string(nlv) + " constraint levels; the kernel holds " +
                                          std::to_string(KR_MAX_LEVELS));
    cnt_per_level.assign(nlv + 1, 0);
    for (int q = 0; q < nc; q++) cnt_per_level[level[q] + 1]++;
    for (int L = 0; L < nlv; L++) cnt_per_level[L + 1] += cnt_per_level[L];
    rec[I_LVL_OFF] = (int)h_lvl.size();
    rec[I_NLV] = nlv;
    for (int L = 0; L <= nlv; L++) h_lvl.push_back(cnt_per_level[L]);
    order.assign(nc, 0);
    {
      std::vector<int> cur(cnt_per_level.begin(), cnt_per_level.end() - 1);
      for (int q = 0; q < nc; q++) order[cur[level[q]]++] = q;  // stable within a level
    }
    rec[I_CON_OFF] = (int)h_cons.size();
    rec[I_NC] = nc;
    for (int s = 0; s < nc; s++) {
      const int k = cl[order[s]];
      const uint32_t *c = cons + 20 * (size_t)k;
      const uint32_t a = (uint32_t)local[c[0]];
      const uint32_t b = c[1] == 0xffffffffu ? 0xffffu : (uint32_t)local[c[1]];
      h_cons.push_back(k);
      h_ab.push_back((int)(a | (b << 16)));
    }
    // collision points in local body order
    rec[I_PT_OFF] = (int)h_pts.size();
    int np = 0;
    for (int j = 0; j < nb; j++) {
      const int g = bl[j];
      const uint32_t off = w->h_coll_range[g], cnt = w->h_coll_range[nB + g];
      h_bpt.push_back(make_int2(np, (int)cnt));
      for (uint32_t q = 0; q < cnt; q++) h_pts.push_back((int)(off + q));
      np += (int)cnt;
    }
    if (np > KR_MAX_ISLAND_COLLPTS)
      return w->fail(KR_ERR_CAPACITY, "connected component " + std::to_string(I) + " has " +
                                          std::to_string(np) + " collision points; the kernel holds " +
                                          std::to_string(KR_MAX_ISLAND_COLLPTS));
    rec[I_NP] = np;
    maxB = std::max(maxB, nb);
    maxC = std::max(maxC, nc);
    maxP = std::max(maxP, np);
    maxLv = std::max(maxLv, nlv);
  }
  cudaError_t e;
  if ((e = dev_upload(&w->d_isl, &w->c_isl, isl)) != cudaSuccess) return w->cuda_fail(e, "upload(islands)");
  if ((e = dev_upload(&w->d_ibodies, &w->c_ibodies, h_bodies)) != cudaSuccess) return w->cuda_fail(e, "upload(island bodies)");
  if ((e = dev_upload(&w->d_icons, &w->c_icons, h_cons)) != cudaSuccess) return w->cuda_fail(e, "upload(island constraints)");
  if ((e = dev_upload(&w->d_iab, &w->c_iab, h_ab)) != cudaSuccess) return w->cuda_fail(e, "upload(island ab)");
  if ((e = dev_upload(&w->d_ipts, &w->c_ipts, h_pts)) != cudaSuccess) return w->cuda_fail(e, "upload(island points)");
  if ((e = dev_upload(&w->d_bpt, &w->c_bpt, h_bpt)) != cudaSuccess) return w->cuda_fail(e, "upload(body point ranges)");
  if ((e = dev_upload(&w->d_lvl, &w->c_lvl, h_lvl)) != cudaSuccess) return w->cuda_fail(e, "upload(levels)");
  w->nI = nI;
  // round up so every per-warp region keeps 16-byte alignment of its arrays
  w->maxB = (maxB + 3) & ~3;
  w->maxC = (maxC + 3) & ~3;
  w->maxP = (maxP + 3) & ~3;
  w->maxLv = maxLv;
  w->smem_bytes =
      sizeof(float) * kWarpsPerBlock * (size_t)warp_smem_words(w->maxB, w->maxC, w->maxP);
  if ((e = cudaFuncSetAttribute(plain_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)w->smem_bytes)) != cudaSuccess)
    return w->cuda_fail(e, "cudaFuncSetAttribute(plain_step_kernel)");
  return KR_OK;
}

}  // namespace

extern "C" int kr_upload(kr_world *w, const float *bodies, const uint32_t *cons, const float *forces,
                         const uint32_t *color_info) {
  if (!w) return KR_ERR_INVALID;
  if (!bodies || (w->nC && !cons)) return w->fail(KR_ERR_INVALID, "kr_upload: null buffer");
  if (color_info) {
    uint32_t acc = 0;
    for (int c = 0; c < 16; c++) {
      if (color_info[c] != acc)
        return w->fail(KR_ERR_INVALID, "colorInfo: colour " + std::to_string(c) +
                                           " does not start where the previous one ends");
      acc += color_info[16 + c];
    }
    if (acc != w->nC)
      return w->fail(KR_ERR_INVALID, "colorInfo covers " + std::to_string(acc) + " of " +
                                         std::to_string(w->nC) + " constraints");
  }
  int rc = build_schedule(w, bodies, cons);
  if (rc != KR_OK) return rc;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(w->d_bodies, bodies, sizeof(float) * 12 * w->nB, cudaMemcpyHostToDevice,
                           w->stream)) != cudaSuccess)
    return w->cuda_fail(e, "upload(bodies)");
  if (w->nC && (e = cudaMemcpyAsync(w->d_cons, cons, sizeof(uint32_t) * 20 * w->nC,
                                    cudaMemcpyHostToDevice, w->stream)) != cudaSuccess)
    return w->cuda_fail(e, "upload(cons)");
  if (forces) {
    if ((e = cudaMemcpyAsync(w->d_forces, forces, sizeof(float) * 4 * w->nB, cudaMemcpyHostToDevice,
                             w->stream)) != cudaSuccess)
      return w->cuda_fail(e, "upload(forces)");
  } else if ((e = cudaMemsetAsync(w->d_forces, 0, sizeof(float) * 4 * w->nB, w->stream)) !=
             cudaSuccess) {
    return w->cuda_fail(e, "upload(forces)");
  }
  if ((e = cudaStreamSynchronize(w->stream)) != cudaSuccess) return w->cuda_fail(e, "upload(sync)");
  w->uploaded = true;
  return KR_OK;
}

namespace {
// Copies the control fields of the 80 B records (packControls, gpuworld.js:331-341).
__global__ void controls_kernel(uint32_t *dst, const uint32_t *src, int nC) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nC) return;
  const uint32_t *s = src + 20 * (size_t)k;
  uint32_t *d = dst + 20 * (size_t)k;
  d[6] = s[6]; d[7] = s[7]; d[8] = s[8]; d[10] = s[10]; d[16] = s[16]; d[17] = s[17];
}
}  // namespace

extern "C" int kr_upload_controls(kr_world *w, const uint32_t *cons) {
  if (!w) return KR_ERR_INVALID;
  if (!w->uploaded) return w->fail(KR_ERR_STATE, "uploadControls before upload");
  if (!w->nC) return KR_OK;
  if (!cons) return w->fail(KR_ERR_INVALID, "kr_upload_controls: null buffer");
  // stage the whole block once, then scatter the six control words per record
  cudaError_t e = cudaMemcpyAsync(w->d_stage, cons, sizeof(uint32_t) * 20 * w->nC,
                                  cudaMemcpyHostToDevice, w->stream);
  if (e != cudaSuccess) return w->cuda_fail(e, "uploadControls(copy)");
  controls_kernel<<<(w->nC + 255) / 256, 256, 0, w->stream>>>(w->d_cons, w->d_stage, (int)w->nC);
  e = cudaGetLastError();
  if (e != cudaSuccess) return w->cuda_fail(e, "uploadControls(scatter)");
  return KR_OK;
}

extern "C" int kr_step(kr_world *w, int32_t n_steps) {
  if (!w) return KR_ERR_INVALID;
  if (!w->uploaded) return w->fail(KR_ERR_STATE, "step before upload");
  if (n_steps < 0) return w->fail(KR_ERR_INVALID, "n_steps < 0");
  if (n_steps == 0 || w->nI == 0) return KR_OK;
  StepArgs A;
  A.K = w->K;
  A.bodies = w->d_bodies;
  A.cons = w->d_cons;
  A.forces = w->d_forces;
  A.coll = w->d_coll;
  A.rects = w->d_rects;
  A.nR = (int)w->nR;
  A.nI = w->nI;
  A.maxB = w->maxB; A.maxC = w->maxC; A.maxP = w->maxP;
  A.T = DeviceTables{w->d_isl, w->d_ibodies, w->d_icons, w->d_iab, w->d_ipts, w->d_bpt, w->d_lvl};
  A.cull_d = w->cull_d;
  A.reach = w->reach;
  const size_t smem = w->smem_bytes;
  cudaError_t e;
  const int grid = (w->nI + kWarpsPerBlock - 1) / kWarpsPerBlock;
  for (int s = 0; s < n_steps; s++) {
    plain_step_kernel<<<grid, 32 * kWarpsPerBlock, smem, w->stream>>>(A);
    e = cudaGetLastError();
    if (e != cudaSuccess) return w->cuda_fail(e, "plain_step_kernel launch");
  }
  return KR_OK;
}

extern "C" int kr_download(kr_world *w, float *bodies, uint32_t *cons) {
  if (!w) return KR_ERR_INVALID;
  if (!w->uploaded) return w->fail(KR_ERR_STATE, "download before upload");
  cudaError_t e;
  if (bodies && (e = cudaMemcpyAsync(bodies, w->d_bodies, sizeof(float) * 12 * w->nB,
                                     cudaMemcpyDeviceToHost, w->stream)) != cudaSuccess)
    return w->cuda_fail(e, "download(bodies)");
  if (cons && w->nC && (e = cudaMemcpyAsync(cons, w->d_cons, sizeof(uint32_t) * 20 * w->nC,
                                            cudaMemcpyDeviceToHost, w->stream)) != cudaSuccess)
    return w->cuda_fail(e, "download(cons)");
  if ((e = cudaStreamSynchronize(w->stream)) != cudaSuccess) return w->cuda_fail(e, "download(sync)");
  return KR_OK;
}

extern "C" int kr_sync(kr_world *w) {
  if (!w) return KR_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) return w->cuda_fail(e, "cudaStreamSynchronize");
  return KR_OK;
}

extern "C" int kr_set_stream(kr_world *w, void *stream) {
  if (!w) return KR_ERR_INVALID;
  cudaError_t e = cudaStreamSynchronize(w->stream);
  if (e != cudaSuccess) return w->cuda_fail(e, "cudaStreamSynchronize");
  if (stream) {
    if (w->own_stream) cudaStreamDestroy(w->stream);
    w->own_stream = false;
    w->stream = static_cast<cudaStream_t>(stream);
  } else if (!w->own_stream) {
    e = cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return w->cuda_fail(e, "cudaStreamCreate");
    w->own_stream = true;
  }
  return KR_OK;
}

extern "C" int kr_world_islands(const kr_world *w, int32_t *n_islands, int32_t *max_levels) {
  if (!w) return KR_ERR_INVALID;
  if (n_islands) *n_islands = w->nI;
  if (max_levels) *max_levels = w->maxLv;
  return KR_OK;
}

extern "C" void kr_destroy(kr_world *w) {
  if (!w) return;
  if (w->stream) cudaStreamSynchronize(w->stream);
  void *ptrs[] = {w->d_bodies, w->d_cons, w->d_stage, w->d_forces, w->d_rects, w->d_coll, w->d_isl,
                  w->d_ibodies, w->d_icons, w->d_iab, w->d_ipts, w->d_lvl, w->d_bpt};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (w->own_stream && w->stream) cudaStreamDestroy(w->stream);
  delete w;
}

// ---------------------------------------------------------------------------
// Allocation-free step (kr_step_noalloc).
//
// For callers that cannot allocate GPU memory -- code running inside a
// host-side memory pool, an embedding that owns every device allocation, a
// real-time loop where cudaMalloc's implicit synchronization is not
// allowed.  Everything the step needs beyond the caller's own buffers (the
// per-creature schedule, the converted rect list, the culling distance)
// lives in one file-scope device array of fixed size, so the call allocates
// nothing on the device or the host.
//
// Scratch layout (words): island records, island bodies, schedule slots,
// slot body pairs, island points, body point ranges, level offsets, rects,
// and the builder's temporaries.  The array is shared by every call on a
// device and keeps the last call's contents; the builder initializes every
// word it reads before reading it.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNaB = KR_NOALLOC_MAX_BODIES;
constexpr int kNaC = KR_NOALLOC_MAX_CONSTRAINTS;
constexpr int kNaP = KR_NOALLOC_MAX_COLLPTS;
constexpr int kNaR = KR_NOALLOC_MAX_RECTS;
// region offsets in words
constexpr int kOffHdr = 0;                                  // n_islands, cull_d, status, pad
constexpr int kOffIsl = 4;
constexpr int kOffBodies = kOffIsl + kNaB * kIslandInts;
constexpr int kOffCons = kOffBodies + kNaB;
constexpr int kOffAb = kOffCons + kNaC;
constexpr int kOffPts = kOffAb + kNaC;
constexpr int kOffBpt = ((kOffPts + kNaP) + 1) & ~1;       // int2, 8-byte aligned
constexpr int kOffLvl = kOffBpt + 2 * kNaB;
constexpr int kOffRects = ((kOffLvl + kNaC + kNaB) + 3) & ~3;  // float4, 16-byte aligned
constexpr int kOffParent = kOffRects + 4 * kNaR;
constexpr int kOffIslandOf = kOffParent + kNaB;
constexpr int kOffLocal = kOffIslandOf + kNaB;
constexpr int kOffRootIsl = kOffLocal + kNaB;
constexpr int kOffCnt = kOffRootIsl + kNaB;                 // kNaB + 1
constexpr int kOffLast = kOffCnt + kNaB + 1;
constexpr int kOffLevel = kOffLast + kNaB;
constexpr int kOffCur = kOffLevel + kNaC;                   // kNaC + 1
constexpr int kScratchWords = kOffCur + kNaC + 1;

static __device__ __align__(256) int g_noalloc_scratch[kScratchWords];

// Single-thread schedule builder: the same islands, bodies, levels, slot
// order and point ranges as build_schedule(), written into the scratch.
__global__ void noalloc_schedule_kernel(int *W, const float *bodies, const uint32_t *cons,
                                        const float *rects, const uint32_t *coll_pts,
                                        const uint32_t *coll_range, int nB, int nC, int nP, int nR) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  int *isl = W + kOffIsl, *ib = W + kOffBodies, *icons = W + kOffCons, *iab = W + kOffAb;
  int *ipts = W + kOffPts, *lvl = W + kOffLvl;
  int2 *bpt = reinterpret_cast<int2 *>(W + kOffBpt);
  float4 *r4 = reinterpret_cast<float4 *>(W + kOffRects);
  int *parent = W + kOffParent, *island_of = W + kOffIslandOf, *local = W + kOffLocal;
  int *root_isl = W + kOffRootIsl, *cnt = W + kOffCnt, *last = W + kOffLast;
  int *level = W + kOffLevel, *cur = W + kOffCur;
  W[kOffHdr + 0] = 0;
  W[kOffHdr + 2] = KR_OK;
  // collRange must tile the points in body order (gpuworld.js:193-199).  The
  // running sum is 64-bit and may never pass nP, so no count can wrap it and
  // every range lies inside [0, nP): the point loops below stay in bounds.
  uint64_t acc = 0;
  for (int g = 0; g < nB; g++) {
    if ((uint64_t)coll_range[g] != acc) { W[kOffHdr + 2] = KR_ERR_INVALID; return; }
    acc += coll_range[nB + g];
    if (acc > (uint64_t)nP) { W[kOffHdr + 2] = KR_ERR_INVALID; return; }
  }
  if (acc != (uint64_t)nP) { W[kOffHdr + 2] = KR_ERR_INVALID; return; }
  for (int g = 0; g < nB; g++) { parent[g] = g; root_isl[g] = -1; }
  for (int k = 0; k < nC; k++) {
    const uint32_t a = cons[20 * (size_t)k], b = cons[20 * (size_t)k + 1];
    if (a >= (uint32_t)nB || (b != 0xffffffffu && b >= (uint32_t)nB)) { W[kOffHdr + 2] = KR_ERR_INDEX; return; }
    if (b != 0xffffffffu) {
      int ra = (int)a, rb = (int)b;
      while (parent[ra] != ra) { parent[ra] = parent[parent[ra]]; ra = parent[ra]; }
      while (parent[rb] != rb) { parent[rb] = parent[parent[rb]]; rb = parent[rb]; }
      if (ra != rb) parent[max(ra, rb)] = min(ra, rb);
    }
  }
  int nI = 0;
  for (int g = 0; g < nB; g++) {
    int r = g;
    while (parent[r] != r) r = parent[r];
    if (root_isl[r] < 0) root_isl[r] = nI++;
    island_of[g] = root_isl[r];
  }
  // bodies per island, ascending
  for (int I = 0; I <= nI; I++) cnt[I] = 0;
  for (int g = 0; g < nB; g++) cnt[island_of[g] + 1]++;
  for (int I = 0; I < nI; I++) cnt[I + 1] += cnt[I];
  for (int I = 0; I < nI; I++) {
    int *rec = isl + I * kIslandInts;
    rec[I_BODY_OFF] = cnt[I];
    rec[I_NB] = cnt[I + 1] - cnt[I];
    if (rec[I_NB] > KR_MAX_ISLAND_BODIES) { W[kOffHdr + 2] = KR_ERR_CAPACITY; return; }
  }
  for (int I = 0; I < nI; I++) cur[I] = cnt[I];
  for (int g = 0; g < nB; g++) {
    const int I = island_of[g];
    local[g] = cur[I] - cnt[I];
    ib[cur[I]++] = g;
  }
  // constraints per island, list order
  for (int I = 0; I <= nI; I++) cnt[I] = 0;
  for (int k = 0; k < nC; k++) cnt[island_of[cons[20 * (size_t)k]] + 1]++;
  for (int I = 0; I < nI; I++) cnt[I + 1] += cnt[I];
  for (int I = 0; I < nI; I++) cur[I] = cnt[I];
  for (int k = 0; k < nC; k++) icons[cur[island_of[cons[20 * (size_t)k]]]++] = k;
  // levels per island, then a stable counting sort of its slots by level
  int lvl_off = 0, pt_off = 0;
  for (int I = 0; I < nI; I++) {
    int *rec = isl + I * kIslandInts;
    const int co = cnt[I], nc = cnt[I + 1] - cnt[I], bo = rec[I_BODY_OFF], nb = rec[I_NB];
    if (nc > KR_MAX_ISLAND_CONSTRAINTS) { W[kOffHdr + 2] = KR_ERR_CAPACITY; return; }
    for (int j = 0; j < nb; j++) last[j] = -1;
    int nlv = 0;
    for (int q = 0; q < nc; q++) {
      const uint32_t *c = cons + 20 * (size_t)icons[co + q];
      const int a = local[c[0]];
      const int b = c[1] == 0xffffffffu ? -1 : local[c[1]];
      int L = last[a] + 1;
      if (b >= 0) L = max(L, last[b] + 1);
      level[q] = L;
      last[a] = L;
      if (b >= 0) last[b] = L;
      nlv = max(nlv, L + 1);
    }
    if (nlv > KR_MAX_LEVELS) { W[kOffHdr + 2] = KR_ERR_CAPACITY; return; }
    int *lv = lvl + lvl_off;
    for (int L = 0; L <= nlv; L++) lv[L] = 0;
    for (int q = 0; q < nc; q++) lv[level[q] + 1]++;
    for (int L = 0; L < nlv; L++) lv[L + 1] += lv[L];
    // stable sort of the island's slots by level; `last` is reused as the
    // per-level cursor (nlv <= KR_MAX_LEVELS < bodies region) and `level`
    // then holds each list position's destination slot
    for (int L = 0; L < nlv; L++) last[L] = lv[L];
    for (int q = 0; q < nc; q++) {
      const int k = icons[co + q];
      const int s = last[level[q]]++;
      // iab holds the final slot's body pair; icons is rewritten after
      const uint32_t *c = cons + 20 * (size_t)k;
      const uint32_t a = (uint32_t)local[c[0]];
      const uint32_t b = c[1] == 0xffffffffu ? 0xffffu : (uint32_t)local[c[1]];
      iab[co + s] = (int)(a | (b << 16));
      level[q] = s;  // destination slot of list position q
    }
    // permute constraint ids into slot order via the `cur` tail as temp
    for (int q = 0; q < nc; q++) cur[q] = icons[co + q];
    for (int q = 0; q < nc; q++) icons[co + level[q]] = cur[q];
    rec[I_CON_OFF] = co;
    rec[I_NC] = nc;
    rec[I_LVL_OFF] = lvl_off;
    rec[I_NLV] = nlv;
    lvl_off += nlv + 1;
    // collision points in local body order; the island's count is checked
    // against the kernel's capacity before any of its points is written
    rec[I_PT_OFF] = pt_off;
    uint64_t np_isl = 0;
    for (int j = 0; j < nb; j++) np_isl += coll_range[nB + ib[bo + j]];
    if (np_isl > (uint64_t)KR_MAX_ISLAND_COLLPTS) { W[kOffHdr + 2] = KR_ERR_CAPACITY; return; }
    int np = 0;
    for (int j = 0; j < nb; j++) {
      const int g = ib[bo + j];
      const uint32_t off = coll_range[g], cn = coll_range[nB + g];
      bpt[bo + j] = make_int2(np, (int)cn);
      for (uint32_t q = 0; q < cn; q++) ipts[pt_off + np + (int)q] = (int)(off + q);
      np += (int)cn;
    }
    rec[I_NP] = np;
    pt_off += np;
  }
  // rects and the culling distance, as kr_create derives them
  double half_thick = 0.0, r_max = 0.0;
  for (int i = 0; i < nR; i++) {
    const float x = rects[4 * i], y = rects[4 * i + 1], rw = rects[4 * i + 2], rh = rects[4 * i + 3];
    r4[i] = make_float4(x, y, x + rw, y + rh);
    const double ht = 0.5 * fmin(fabs((double)rw), fabs((double)rh));
    half_thick = isfinite(ht) ? fmax(half_thick, ht) : HUGE_VAL;
  }
  for (int i = 0; i < nP; i++) {
    const float r = __uint_as_float(coll_pts[4 * i + 3]);
    r_max = isfinite(r) ? fmax(r_max, fabs((double)r)) : HUGE_VAL;
  }
  const double cull = fmax(r_max, half_thick) + 2.0 + kr::kCullSlack + 1.0;
  reinterpret_cast<float *>(W)[kOffHdr + 1] = (isfinite(cull) && cull < 1e30) ? (float)cull : 1e30f;
  W[kOffHdr + 0] = nI;
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock) noalloc_step_kernel(StepArgs A, const int *W) {
  StepArgs B = A;
  B.nI = W[kOffHdr + 0];
  B.cull_d = reinterpret_cast<const float *>(W)[kOffHdr + 1];
  if (W[kOffHdr + 2] != KR_OK) return;
  plain_step_body(B);
}

int g_noalloc_status_host = 0;
void *g_noalloc_ptr[64] = {nullptr};

}  // namespace

extern "C" int kr_step_noalloc(const kr_solver_params *params, uint32_t n_bodies, uint32_t n_constraints,
                               float *bodies, uint32_t *cons, float *forces, const float *rects,
                               uint32_t n_rects, const uint32_t *coll_pts, uint32_t n_coll_pts,
                               const uint32_t *coll_range, int32_t n_steps, void *stream) {
  if (!params || !bodies || !forces || !rects || !coll_range || (n_constraints && !cons) ||
      (n_coll_pts && !coll_pts) || n_steps < 0)
    return KR_ERR_INVALID;
  // The kernels move bodies, forces, constraints and collision points as
  // 16-byte vectors and read rects and collRange as 4-byte words; a caller's
  // pool may hand out any address, so misaligned buffers are refused here,
  // before the device is touched.
  auto misaligned = [](const void *q, uintptr_t a) { return (reinterpret_cast<uintptr_t>(q) & (a - 1)) != 0; };
  if (misaligned(bodies, 16) || misaligned(forces, 16) || (cons && misaligned(cons, 16)) ||
      (coll_pts && misaligned(coll_pts, 16)) || misaligned(rects, 4) || misaligned(coll_range, 4))
    return KR_ERR_INVALID;
  const kr_solver_params &p = *params;
  const float hf = static_cast<float>(p.h);
  if (!(p.iterations >= 1 && p.iterations <= 64) || !(p.substeps >= 1 && p.substeps <= 64) ||
      !(hf > 0.f && hf < 1.f) || n_bodies < 1 || n_rects < 1)
    return KR_ERR_INVALID;
  if (n_bodies > (uint32_t)kNaB || n_constraints > (uint32_t)kNaC || n_coll_pts > (uint32_t)kNaP ||
      n_rects > (uint32_t)kNaR)
    return KR_ERR_CAPACITY;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return KR_ERR_CUDA;
  // set-up once per device, with that device current: the device address of
  // the scratch array (its host-side name is only a stand-in)
  if (!g_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) return KR_ERR_CUDA;
    g_noalloc_ptr[dev] = ptr;
  }
  int *W = static_cast<int *>(g_noalloc_ptr[dev]);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_steps == 0) return KR_OK;
  noalloc_schedule_kernel<<<1, 32, 0, st>>>(W, bodies, cons, rects, coll_pts, coll_range,
                                           (int)n_bodies, (int)n_constraints, (int)n_coll_pts,
                                           (int)n_rects);
  if (cudaGetLastError() != cudaSuccess) return KR_ERR_CUDA;
  // the builder's verdict decides the return code (a 4-byte copy into static
  // host memory, which also orders this call after the builder)
  if (cudaMemcpyAsync(&g_noalloc_status_host, W + kOffHdr + 2, sizeof(int), cudaMemcpyDeviceToHost,
                      st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return KR_ERR_CUDA;
  if (g_noalloc_status_host != KR_OK) return g_noalloc_status_host;
  StepArgs A;
  A.K.h = hf;
  A.K.invH = static_cast<float>(1.0 / p.h);
  A.K.invH2 = static_cast<float>(1.0 / (p.h * p.h));
  const float nl = -static_cast<float>(p.lin_drag), na = -static_cast<float>(p.ang_drag);
  A.K.linDamp = static_cast<float>(std::exp(static_cast<double>(nl * hf)));
  A.K.angDamp = static_cast<float>(std::exp(static_cast<double>(na * hf)));
  A.K.maxSpeed = static_cast<float>(p.max_speed);
  A.K.maxAngSpeed = static_cast<float>(p.max_ang_speed);
  A.K.substeps = p.substeps;
  A.K.iterations = p.iterations;
  A.bodies = bodies;
  A.cons = cons;
  A.forces = forces;
  A.coll = reinterpret_cast<const uint4 *>(coll_pts);
  A.rects = reinterpret_cast<const float4 *>(W + kOffRects);
  A.nR = (int)n_rects;
  A.cull_d = 0.f;
  A.reach = -1.f;
  A.nI = 0;
  // shared memory for the largest island the world can hold
  A.maxB = ((int)std::min<uint32_t>(n_bodies, KR_MAX_ISLAND_BODIES) + 3) & ~3;
  A.maxC = ((int)std::min<uint32_t>(std::max<uint32_t>(n_constraints, 1), KR_MAX_ISLAND_CONSTRAINTS) + 3) & ~3;
  A.maxP = ((int)std::min<uint32_t>(std::max<uint32_t>(n_coll_pts, 1), KR_MAX_ISLAND_COLLPTS) + 3) & ~3;
  A.T = DeviceTables{W + kOffIsl, W + kOffBodies, W + kOffCons, W + kOffAb, W + kOffPts,
                     reinterpret_cast<const int2 *>(W + kOffBpt), W + kOffLvl};
  const size_t smem = sizeof(float) * kWarpsPerBlock * (size_t)warp_smem_words(A.maxB, A.maxC, A.maxP);
  if (cudaFuncSetAttribute(noalloc_step_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return KR_ERR_CUDA;
  const int grid = ((int)n_bodies + kWarpsPerBlock - 1) / kWarpsPerBlock;  // islands <= bodies
  for (int s = 0; s < n_steps; s++) {
    noalloc_step_kernel<<<grid, 32 * kWarpsPerBlock, smem, st>>>(A, W);
    if (cudaGetLastError() != cudaSuccess) return KR_ERR_CUDA;
  }
  return KR_OK;
}
