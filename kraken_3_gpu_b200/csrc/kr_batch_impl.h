// kr_batch_impl.h -- host-side internals of the batched engine, shared by
// kr_batch.cu (the engine and its kernel) and kr_serve.cu (the rollout
// server built on the engine's slots).  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/kraken_batch.h"
#include "kr_solver.cuh"
#include "kr_template.h"

namespace krb {

constexpr int kMaxW = 16;                                      // warps per CTA
constexpr int kMaxCPC = 64;                                    // creatures per CTA (W * 32 / G)
constexpr int kBodyPad = 76;                                   // >= kMaxTplBodies, /4
constexpr int kStateStride = 6 * kBodyPad;                     // px py vx vy ang av
constexpr int kCtrlStride = KR_BATCH_MAX_ARMS * (KR_BATCH_MAX_SEGS + 1);  // 80

// Template record on the device: sizes and offsets into the flat arrays.
// Constraint slots, level offsets and arm grip slots exist once per solve
// schedule (kr::schedule_index of the lanes per creature).
struct TplDev {
  int nb, nc, np, arms, segs;
  int nlv[kr::kSchedules];
  float r_max;
  float off_max;   // largest distance of a collision point from its body's centre
  double reach;
  int o_b, o_p, o_a, o_s;
  int o_c[kr::kSchedules], o_l[kr::kSchedules], o_g[kr::kSchedules];
};

struct TplArrays {
  const float *im, *ii;
  const int *boff, *bcnt;
  const int *ab, *type, *motor, *garm;
  const float *lax, *lay, *lbx, *lby, *rest, *minA, *maxA;
  const int *lvl;
  const float *plx, *ply, *pr;
  const int *pbody;
  const int *arm_tip, *arm_grip, *arm_seg0, *arm_segs;  // arm_grip: per schedule
};

// Per-slot record (device resident; the host keeps a mirror of the static
// fields).
struct SlotMeta {
  int tpl, map, horizon, step;
  uint32_t rng;
  float comp;       // muscle compliance (f32 as packControls writes it)
  float tone;
  int attach_events;  // arms newly anchored after a step
  int ctrl;         // KR_CTRL_* of this slot
  int pad;          // the rollout server's request tag (BatchArgs::tag_done)
  double prev_vx, prev_vy;
  double path_len;
  double last_x, last_y;
  // postStep accumulators, core.js:297-356
  double tone_d, spawn_x, spawn_y, spawn_reach;
  double angular_accum, forward_prog, grip_pull_prog, spawn_dist_max, free_move, energy, max_disp;
  int anchored_steps, grip_cycles, strides;
  unsigned arm_anchored;  // bit a: arm a anchored after the last step; bit 8: any
};

// policy parameters of an arms x segs body (kraken_batch.h layout: W1
// 64 x (n_in + 1) then W2 n_out x 65, row-major, bias last)
__host__ __device__ inline int policy_param_count(int arms, int segs) {
  return KR_POLICY_HIDDEN * (6 * arms + 7) + (arms * segs + arms) * (KR_POLICY_HIDDEN + 1);
}

// position of public parameter p in the device layout, the transposes
// W1T (n_in + 1) x 64 and W2T 65 x n_out (lanes then read consecutive words)
__host__ __device__ inline int policy_device_index(int arms, int segs, int p) {
  const int n_in = 6 * arms + 6, n_out = arms * segs + arms, H = KR_POLICY_HIDDEN;
  if (p < H * (n_in + 1)) return (p % (n_in + 1)) * H + p / (n_in + 1);
  const int q = p - H * (n_in + 1);
  return H * (n_in + 1) + (q % (H + 1)) * n_out + q / (H + 1);
}

// makeSdf's distance (src/world/map.js:91-118) in f64 over rects x y w h:
// false where the JS returns null (no finite winner).  Host and device run
// this same code (IEEE f64 add, multiply and sqrt; min / max as std::min /
// std::max).
__host__ __device__ inline bool sdf64(const double *rects, int n, double px, double py, double *out) {
  double best = INFINITY, thr = INFINITY;  // thr = best * best, the JS's per-rect product
  const double *r = rects;
  for (int i = 0; i < n; i++, r += 4) {
    const double xr = r[0] + r[2], yb = r[1] + r[3];
    const double mx = xr < px ? xr : px, my = yb < py ? yb : py;
    const double cx = r[0] < mx ? mx : r[0], cy = r[1] < my ? my : r[1];
    const double dx = px - cx, dy = py - cy, d2 = dx * dx + dy * dy;
    if (d2 > 1e-12) {
      if (d2 < thr) {
        best = sqrt(d2);
        thr = best * best;
      }
    } else {
      const double a = px - r[0], b = xr - px, e = py - r[1], f = yb - py;
      const double ab = b < a ? b : a, ef = f < e ? f : e, m = ef < ab ? ef : ab;
      if (-m < best) {
        best = -m;
        thr = best * best;
      }
    }
  }
  if (!(best < INFINITY && best > -INFINITY)) return false;
  *out = best;
  return true;
}

// measureReach (src/sim/fitness.js:74-88) along one ray from (x, y) with
// direction (c, s): march in 12 px steps while the makeSdf distance stays
// positive, up to 3.5 reach; the distance marched.
__host__ __device__ inline double reach_ray(const double *rects, int n, double reach, double x, double y,
                                            double c, double s) {
  double d = 0;
  while (d < reach * 3.5) {
    d += 12;
    double h;
    if (!sdf64(rects, n, x + c * d, y + s * d, &h) || h <= 0) break;
  }
  return d;
}

// raymarch, src/senses/echo.js:94-110: the distance to the first surface
// along the ray (cx, cy) = (cos, sin) of its angle, adaptive steps, at most
// 96, maxd when nothing is hit
__host__ __device__ inline double echo_march(const double *rects, int n, double x, double y, double cx,
                                             double cy, double maxd) {
  double t = 0;
  for (int i = 0; i < 96; i++) {
    if (t >= maxd) return maxd;
    double d;
    if (!sdf64(rects, n, x + cx * t, y + cy * t, &d)) return maxd;
    if (d <= 0) return t;
    const double adv = d * 0.85;
    t += adv > 1.0 ? adv : 1.0;
    if (d < 0.5) return t;
  }
  return maxd;
}

// Env steps of the light-position table of an engine with n_lights map
// lights: a map's lights move by the sim's clock alone (tickMapLights), so
// every creature of a map sees the same positions after its step t, and the
// engine tabulates them once (16 bytes per light and step, at most 64 MB,
// at most 4,096 steps; later steps move the lights per creature as before).
inline int light_table_steps(long n_lights) {
  if (n_lights <= 0) return 0;
  const long cap = (64L << 20) / (16L * n_lights);
  return (int)(cap < 4096 ? cap : 4096);
}

// net.js weightCount for an arms-armed body: n_in = 10 arms + 45 inputs,
// KR_NET_HIDDEN twice, 3 arms + 2 outputs
__host__ __device__ inline int net_inputs(int arms) { return 10 * arms + 45; }
__host__ __device__ inline int net_outputs(int arms) { return 3 * arms + 2; }
__host__ __device__ inline int net_param_count(int arms) {
  const int ni = net_inputs(arms), no = net_outputs(arms), H = KR_NET_HIDDEN;
  return ni * H + H + H * H + H + H * no + no;
}

// Device layout of a net genome: the blocks of net.js's layout at the same
// offsets (W1 | b1 | W2 | unread | W3 | b3, forwardInto's b1..b5), each
// weight matrix transposed (input-major, so the lanes of one input read
// consecutive words) and the unread block replaced by the layer-2 bias as
// forwardInto reads it, w[b2 + j] -- which is also W2's first row.  Public
// parameter p goes to *d0 and, for that first row, also to *d1; returns the
// number of places (0 for the unread block).
__host__ __device__ inline int net_device_slots(int arms, int p, int *d0, int *d1) {
  const int ni = net_inputs(arms), no = net_outputs(arms), H = KR_NET_HIDDEN;
  const int b1 = ni * H, b2 = b1 + H, b3 = b2 + H * H, b4 = b3 + H, b5 = b4 + H * no;
  if (p < b1) { *d0 = (p % ni) * H + p / ni; return 1; }
  if (p < b2) { *d0 = p; return 1; }
  if (p < b3) {
    const int q = p - b2;
    *d0 = b2 + (q % H) * H + q / H;
    if (q < H) { *d1 = b3 + q; return 2; }
    return 1;
  }
  if (p < b4) return 0;
  if (p < b5) { const int q = p - b4; *d0 = b4 + (q % H) * no + q / H; return 1; }
  *d0 = p;
  return 1;
}

// echo.js constants (ECHO_RANGE, SOUND_SPEED, ECHO_INTERVAL) and the
// pending-echo capacity: an echo arrives within 2 range / speed = 0.756 s of
// its emission and emissions are at least 0.42 s apart, so at most two
// emissions (24 echoes) are pending at once
constexpr double kEchoRange = 340.0, kEchoSpeed = 900.0, kEchoInterval = 0.42;
constexpr int kEchoPending = 32;

// Per-slot state of KR_CTRL_NET (f64 where the reference keeps f64 state;
// values the trainer only reads through its Float32Array input are kept in
// f32): the sim time (sim.time and map.t advance alike), the echo (cooldown,
// pending echoes sorted by arrival, last arrived range / intensity per ray),
// the creature's copy of its map's lights, the light and contact senses,
// and the network's last input, hidden and output vectors.
struct NetRec {
  double time, cooldown;
  double contact[KR_BATCH_MAX_ARMS];
  double light_xy[2 * KR_NET_MAX_LIGHTS];
  double p_at[kEchoPending];
  double ray_d[KR_NET_RAYS];
  float p_range[kEchoPending], p_inten[kEchoPending];
  int p_ray[kEchoPending];
  float range[KR_NET_RAYS], inten[KR_NET_RAYS];
  float light_v[4];          // left, right, total
  double lc[3 * KR_NET_MAX_LIGHTS];  // per sample point and light: its contribution
  int n_pending, emit_count, wants_emit, dropped;
  float x[KR_NET_IN_STRIDE];
  float h[2 * KR_NET_HIDDEN];
  float out[KR_NET_OUT_STRIDE];
};

// the 16 ray directions of measureReach, angle k / 16 * 2 pi, from the host's libm
struct RayDirs {
  double c[16], s[16];
};

// A set of slots launched together on one stream: every slot (the public
// engine calls) or an explicit list (the rollout server's partitions).
struct Part {
  bool all = true;
  std::vector<int> slots;
  int *d_groups = nullptr;        // n_groups x cpc slot ids
  size_t c_groups = 0;
  int *h_groups = nullptr;        // pinned staging of the groups
  size_t ch_groups = 0;
  int n_groups = 0;
  bool dirty = true;
  int *d_queue = nullptr;         // work-queue counter
  cudaStream_t stream = nullptr;  // the engine's stream when null
  const int *stop = nullptr;      // device word: non-zero ends the launch early (see BatchArgs::stop)
  int *tag_done = nullptr;        // per tag (SlotMeta::pad): creatures that reached their horizon
  cudaEvent_t staged = nullptr;   // the groups' host-to-device copy has run
  bool staged_pending = false;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // launch timing
  uint64_t h2d_bytes = 0;         // group uploads so far
  // the live slots with their template, remaining steps and control mode,
  // gathered in one pass over the slot records (gather_live) and used by
  // the next build_groups; then the launch order's scratch
  std::vector<int> g_live, g_tpl, g_rem, g_ctrl, s_live, perm, perm2;
  std::vector<uint64_t> keys, keys2;
  long g_per_arm = 0, g_net = 0;   // live slots under the policy or the net / under the net
  bool gathered = false;
};

// slot data a spawn writes, built on the host
struct SpawnInit {
  std::vector<float> pose;       // n x kStateStride
  std::vector<SlotMeta> meta;    // n
};

}  // namespace krb

struct kr_batch {
  kr_batch_desc d{};
  kr::SolverConsts K{};
  std::string err;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int capacity = 0, n_maps = 0;
  // templates
  std::vector<kr::Template> tpls;
  std::map<std::pair<int, int>, int> tpl_index;
  std::vector<krb::TplDev> h_tpl;
  krb::TplDev *d_tpl = nullptr;
  void *d_tpl_arrays[23] = {nullptr};
  krb::TplArrays T{};
  // maps
  float4 *d_rects = nullptr;
  int *d_map_off = nullptr;
  float *d_map_cull = nullptr;
  std::vector<float> h_map_cull;
  std::vector<double> h_rects;         // every map's rects x y w h as the device holds them
  std::vector<int> h_map_off;
  double *d_rects64 = nullptr;         // h_rects on the device (measureReach, senses)
  krb::RayDirs rays{};
  // KR_CTRL_NET: lights per map (x y r ir ph sp), offsets, sizes; per-slot state
  double *d_lights = nullptr;
  int *d_light_off = nullptr;
  double *d_map_size = nullptr;
  double2 *d_light_tab = nullptr;      // per light, its position after env step t < light_T
  int light_T = 0;
  krb::NetRec *d_net = nullptr, *s_net = nullptr;
  std::vector<int> h_pw_arms;          // arms of each net individual (-1: unused)
  // slots
  float *d_state = nullptr;
  float4 *d_grip = nullptr;
  float2 *d_glam = nullptr;
  double2 *d_cd = nullptr;           // per arm: reflex cooldown, f64 break force
  float *d_ctrl = nullptr;
  krb::SlotMeta *d_meta = nullptr;
  float *d_obs = nullptr;
  std::vector<krb::SlotMeta> h_meta;   // host mirror of tpl / map / horizon (step on device)
  std::vector<int> h_remaining;        // remaining steps as of the last schedule
  // the partition of every slot (public engine calls)
  krb::Part main;
  // snapshot of every slot (kr_batch_snapshot / kr_batch_restore)
  float *s_state = nullptr;
  float4 *s_grip = nullptr;
  float2 *s_glam = nullptr;
  double2 *s_cd = nullptr;
  float *s_ctrl = nullptr;
  krb::SlotMeta *s_meta = nullptr;
  std::vector<int> s_remaining;
  int *s_groups = nullptr;        // groups built for the snapshot state
  int s_n_groups = -1, s_cpc = 0, s_G = 0;
  // launch shape
  int G = 16, W = 8, ctas_per_sm = 0, n_sm = 0;
  int unroll = 1;               // unroll factor of the kernel's substep loop (1 or 2)
  int smem_per_sm = 0, smem_reserved = 0, smem_optin = 0;
  bool auto_shape = true;       // until kr_batch_set_launch: G and W from the live count
  int cpc = 16;                 // creature entries per group: W * 32 / G
  std::vector<int> tpl_cpg;     // creatures per group of each template
  size_t smem_dyn = 0;          // dynamic shared memory per CTA
  bool shape_dirty = true;
  // policy: pw_stride floats per individual (device layout), individual of
  // each slot, the body shape each individual's weights are laid out for
  float *d_pw = nullptr;
  int *d_pw_idx = nullptr;
  size_t pw_capacity = 0;
  int pw_stride = 0, n_individuals = 0;
  std::vector<int> h_pw_idx, h_pw_tpl;
  // time-sliced runs (kr_batch_set_slice)
  float slice_ms = 0.f;
  bool slice_ready = false;            // the buffers below exist
  int *d_stop = nullptr;               // the kernel's stop word
  int *h_flag = nullptr;               // pinned {0, 1}: the values it is set to
  int *d_steps = nullptr, *h_steps = nullptr;  // every slot's step counter after a slice
  cudaStream_t ctl = nullptr;          // the stop word's copy while a slice runs
  cudaEvent_t slice_start = nullptr, slice_end = nullptr;
  int last_slices = 0, last_kernels = 0;  // of the last kr_batch_run
  long long last_creature_launches = 0;    // ... live creatures per slice, summed

  int fail(int code, const std::string &m) { err = m; return code; }
  int cuda_fail(cudaError_t e, const char *what) {
    err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return KR_ERR_CUDA;
  }
};

namespace krb {

// template id of an arms x segs body (built on first use), -1 if out of range
int ensure_template(kr_batch *b, int arms, int segs);
// (re)uploads every template; call after ensure_template added one
int upload_templates(kr_batch *b);
// creatures per group of every template and the CTA's shared memory
int plan_shape(kr_batch *b);
// lanes per creature the automatic launch shape gives `live` creatures, of
// which `per_arm` run the policy or net controller (their proprioception
// and controller run per arm)
int auto_lanes(const kr_batch *b, long live, long per_arm);
// the part's live slots (remaining steps > 0) with their template, remaining
// steps and control mode, in slot-list order, into p.g_*
void gather_live(kr_batch *b, Part &p);
// groups of the part's live slots, longest work first, staged to the device
int build_groups(kr_batch *b, Part &p, int max_steps);
// one persistent launch over the part's groups, min(max_steps, remaining)
// env steps per slot; asynchronous on the part's stream
int launch_part(kr_batch *b, Part &p, int max_steps, bool timed);
// host-side initial data of n creatures into pose (n x kStateStride f32,
// every word written) and meta (n records); ctrl: per-creature control mode
// (NULL: ctrl_mode for all).  Fails on a bad body shape, map or horizon.
int prepare_spawn_into(kr_batch *b, int n, const int32_t *arms, const int32_t *segs, const int32_t *map_id,
                       const double *x, const double *y, const double *angle, const int32_t *horizon,
                       const uint32_t *control_seed, const float *tone, int ctrl_mode, const int32_t *ctrl,
                       float *pose, SlotMeta *meta, int *first_bad);
// host-side initial data of n creatures (spawn pose, meta); fails on a bad
// body shape or map
int prepare_spawn(kr_batch *b, int n, const int32_t *arms, const int32_t *segs, const int32_t *map_id,
                  const double *x, const double *y, const double *angle, const int32_t *horizon,
                  const uint32_t *control_seed, const float *tone, int ctrl_mode, SpawnInit *out,
                  int *first_bad);
// writes prepared creatures into the given slots (device copies of the
// pose / meta / slot arrays), asynchronous on `stream`
cudaError_t launch_spawn(kr_batch *b, const int *d_slots, const float *d_pose, const SlotMeta *d_meta,
                         int n, cudaStream_t stream);
cudaStream_t part_stream(const kr_batch *b, const Part &p);
// the metrics record of a slot (kraken_batch.h, KR_METRIC_WORDS), score included
void slot_metrics(const SlotMeta &m, double *out);
// public -> device layout of one individual's policy parameters
void transpose_policy(const float *pub, int arms, int segs, float *dev);
void free_part(Part &p);

}  // namespace krb
