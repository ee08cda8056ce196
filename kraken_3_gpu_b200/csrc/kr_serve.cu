// kr_serve.cu -- the rollout server (include/kraken_serve.h) on the batched
// engine's slots.
//
// Scheduling.  The slots are split into two partitions, each with its own
// stream.  A round of partition p: wait for p's previous round (partition
// 1 - p keeps the GPU busy meanwhile), complete the requests that ended in
// it, admit arrived requests (FIFO) into free slots of p, stage their spawn
// and policy weights, and launch chunk_steps env steps of every creature of
// p (the engine's persistent kernel over groups of one template, largest
// work first).  Rounds alternate between the partitions, so one
// partition's launch is queued behind the other's and fills its tail.
//
// A request's completion round is known when it is admitted (every creature
// advances min(chunk, remaining) steps per round), so the results of the
// requests ending in a round are gathered on the device and copied back in
// that round, with no extra synchronization.
//
// Policy weights: theta + sigma * eps (even individuals) and theta - sigma *
// eps (odd), eps from a counter-based generator -- splitmix64 (Steele, Lea,
// Flood 2014) of (seed, pair, parameter) gives two 24-bit uniforms, Box-Muller
// gives the normal -- so every individual's weights are a pure function of
// the request and the device needs no generator state.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <deque>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/kraken_serve.h"
#include "kr_batch_impl.h"

namespace {
using namespace krb;

constexpr int kMaxParams = KR_POLICY_HIDDEN * (6 * KR_BATCH_MAX_ARMS + 7) +
                           (KR_BATCH_MAX_ARMS * KR_BATCH_MAX_SEGS + KR_BATCH_MAX_ARMS) * (KR_POLICY_HIDDEN + 1);
constexpr int kMaxNetParams = ((10 * KR_BATCH_MAX_ARMS + 45) * KR_NET_HIDDEN + 2 * KR_NET_HIDDEN +
                               KR_NET_HIDDEN * KR_NET_HIDDEN + (3 * KR_BATCH_MAX_ARMS + 2) * (KR_NET_HIDDEN + 1) + 3) &
                              ~3;  // net.js genome of the largest body, 16-byte multiple
constexpr int kMaxThetaPerRound = 64;   // policy requests admitted into one partition per round
constexpr uint64_t kFixedBytes = 8ull << 20;  // tables, maps, queues, events

thread_local std::string g_serve_error;

__host__ __device__ inline uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// standard normal number `p` of mirrored pair `pair` of a request
__device__ inline float eps_normal(uint64_t seed, int pair, int p) {
  const uint64_t x = splitmix64(seed ^ splitmix64(((uint64_t)(uint32_t)pair << 32) | (uint32_t)p));
  const double u1 = ((double)(x >> 40) + 1.0) * (1.0 / 16777216.0);  // (0, 1]
  const double u2 = (double)(x & 0xffffffULL) * (1.0 / 16777216.0);  // [0, 1)
  return (float)(sqrt(-2.0 * log(u1)) * cospi(2.0 * u2));
}

__global__ void eps_kernel(uint64_t seed, int pair, int n, float *out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = eps_normal(seed, pair, p);
}

struct PJob {
  int slot, theta_off, arms, segs, pair;
  float sign, sigma;
  uint64_t seed;
};

// weights of newly admitted individuals: theta +- sigma * eps for public
// parameter p, stored at its place(s) in the device layout of the fused
// policy or, with net, of the reference net (net_device_slots)
__global__ void perturb_kernel(float *w, int stride, const float *theta, const PJob *jobs, int n, int net) {
  if ((int)blockIdx.x >= n) return;
  const PJob j = jobs[blockIdx.x];
  float *dst = w + (size_t)j.slot * stride;
  const float *th = theta + j.theta_off;
  const int np = net ? net_param_count(j.arms) : policy_param_count(j.arms, j.segs);
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    const float d = __fmul_rn(j.sigma, eps_normal(j.seed, j.pair, p));
    const float v = __fadd_rn(th[p], j.sign < 0.f ? -d : d);
    if (!net) {
      dst[policy_device_index(j.arms, j.segs, p)] = v;
      continue;
    }
    int d0 = 0, d1 = 0;
    const int k = net_device_slots(j.arms, p, &d0, &d1);
    if (k > 0) dst[d0] = v;
    if (k > 1) dst[d1] = v;
  }
}

// the records of the creatures in slots[0..n) (results are derived on the host)
__global__ void gather_kernel(const SlotMeta *meta, const int *slots, int n, SlotMeta *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = meta[slots[i]];
}

// the completion count of every request admitted in a staging starts at 0:
// its tag (the request's first slot) may have counted an earlier request
__global__ void clear_done_kernel(const SlotMeta *meta, const int *slots, int n, int *done) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && meta[i].pad == slots[i]) done[slots[i]] = 0;
}

// every slot's step counter into one contiguous array (read back after a slice)
__global__ void steps_kernel(const SlotMeta *meta, int n, int *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = meta[i].step;
}

struct Req {
  int64_t id = 0;
  kr_request r{};
  std::vector<float> theta;
  std::vector<double> xs, ys, angles;   // per individual (empty: common pose)
  std::vector<uint32_t> seeds;          // per individual control streams
  int part = -1;
  std::vector<int> slots;
  int rounds_left = 0;
  double arrival = 0, admitted = -1, completed = -1;
  std::vector<double> results;
  int pending = 0;                      // sliced scheduling: creatures not yet at their horizon
  int64_t seq = 0;                      // admission order
  bool done = false;
  bool holding = false;                 // its slots are still its own (a request completed while its
                                        // slice runs keeps them until the slice ends)
  bool release_pending = false;         // released while holding: erased when its slots are freed
};

// admission's per-creature inputs, reused between admissions
struct AdmitScratch {
  std::vector<Req *> reqs;
  std::vector<int32_t> arms, segs, maps, hor, ctrl;
  std::vector<double> xs, ys, an;
  std::vector<uint32_t> seeds;
  std::vector<float> tones;
};

// staging of one partition (pinned host + device), reused every round
struct Stage {
  float *h_pose = nullptr, *d_pose = nullptr;      // part_cap x kStateStride
  SlotMeta *h_meta = nullptr, *d_meta = nullptr;   // part_cap
  int *h_slots = nullptr, *d_slots = nullptr;      // part_cap
  PJob *h_jobs = nullptr, *d_jobs = nullptr;       // part_cap
  float *h_theta = nullptr, *d_theta = nullptr;    // kMaxThetaPerRound x kMaxParams
  int *h_rslots = nullptr, *d_rslots = nullptr;    // part_cap
  SlotMeta *h_res = nullptr, *d_res = nullptr;     // part_cap records of completing slots
};

struct Round {
  bool inflight = false;
  cudaEvent_t done = nullptr;
  std::vector<Req *> completing;
  bool timed = false;
};

// weights per slot: the fused policy's or the reference net's largest body
int weight_stride(const kr_server_desc &d) { return d.net ? kMaxNetParams : kMaxParams; }

uint64_t slot_bytes(const kr_server_desc &d) {
  uint64_t b = (uint64_t)kStateStride * 4 + KR_BATCH_MAX_ARMS * (16 + 8 + 8) + (uint64_t)kCtrlStride * 4 +
               sizeof(SlotMeta);
  b += (uint64_t)d.obs_ring * KR_OBS_STRIDE * 4;
  if (d.policy) b += (uint64_t)kMaxParams * 4 + 4;
  if (d.net) b += (uint64_t)kMaxNetParams * 4 + 4 + sizeof(NetRec);
  // partition staging and work groups (two partitions of half the slots, or
  // one of all slots), and a slice's step-counter readback
  b += (uint64_t)kStateStride * 4 + sizeof(SlotMeta) + 4 + sizeof(PJob) + 4 + sizeof(SlotMeta) + 2 * 4;
  if (d.slice_ms > 0) b += 8;  // step readback, per-request completion count
  return b;
}

uint64_t fixed_bytes(const kr_server_desc &d) {
  uint64_t b = kFixedBytes;
  if (d.n_maps > 0 && d.map_rect_off) b += (uint64_t)d.map_rect_off[d.n_maps] * 16 + (uint64_t)d.n_maps * 8;
  if (d.policy || d.net) b += 2ull * kMaxThetaPerRound * weight_stride(d) * 4;
  if (d.net && d.lights && d.map_light_off) {
    const long nl = d.map_light_off[d.n_maps];
    b += (uint64_t)nl * 48 + (uint64_t)d.n_maps * 20 + (uint64_t)nl * light_table_steps(nl) * 16;
  }
  return b;
}

}  // namespace

struct kr_server {
  kr_server_desc d{};
  kr_batch *b = nullptr;
  Part parts[2];
  Stage stage[2];
  Round round[2];
  cudaStream_t streams[2] = {nullptr, nullptr};
  // running requests per partition, in admission order (a running request
  // cannot be released, so its map entry, and the pointer, stay valid)
  std::vector<Req *> active[2];
  std::vector<Req *> slot_req;   // the request holding each slot
  int part_used[2] = {0, 0};
  int next = 0;
  int capacity = 0, part_cap = 0, chunk = 1;
  uint64_t bytes_per_slot = 0, device_bytes = 0;
  std::deque<int64_t> queue;
  AdmitScratch adm;
  std::unordered_map<int64_t, Req> reqs;
  std::vector<int> free_slots;
  std::vector<int64_t> done_ids;
  int64_t next_id = 1;
  int64_t submitted = 0, admitted = 0, completed = 0, rounds = 0;
  double creature_steps = 0, device_ms = 0;
  uint64_t h2d_bytes = 0, d2h_bytes = 0;
  std::chrono::steady_clock::time_point t0;
  // sliced scheduling (slice_ms > 0): one partition, preemptible slices
  bool sliced = false;
  double slice_s = 0;            // the time slice (slice_ms)
  int *d_stop = nullptr;          // the kernel's stop word
  int *h_flag = nullptr;          // pinned {0, 1}: the values the stop word is set to
  int *h_steps = nullptr;         // pinned: every slot's step counter after a slice
  int *d_steps = nullptr;
  cudaStream_t ctl = nullptr;     // the stop word's and completion counts' copies while a slice runs
  cudaEvent_t staged = nullptr;   // a slice's admissions done: the control stream waits for it
  double slice_t0 = 0;
  bool stop_sent = false;
  int *d_done = nullptr;          // per request tag (its first slot): creatures that reached their horizon
  int *h_done = nullptr;          // pinned copy of d_done, polled while a slice runs
  std::vector<int> prev_done;     // h_done as of the poll before
  std::vector<int> gather_slots;  // slots whose records a poll copies back
  std::vector<int> rec_pos;       // ... and where each record lands in the staging
  double polled = -1;             // server time of the last poll
  long done_unfreed = 0;          // slots of requests completed while their slice runs
  double gap_s = 0;               // host time between a slice's end and the next launch (running mean)
  double gap_sum = 0;             // ... summed
  std::string err;

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  int fail(int code, const std::string &m) { err = m; return code; }
  int cuda_fail(cudaError_t e, const char *what) {
    err = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
    return KR_ERR_CUDA;
  }
  int batch_fail(int rc) {
    err = std::string("engine: ") + kr_batch_last_error(b);
    return rc;
  }
};

namespace {

int check_desc(const kr_server_desc *d, std::string *why) {
  if (!d) { *why = "null descriptor"; return KR_ERR_INVALID; }
  if (d->chunk_steps < 1 || d->chunk_steps > 1 << 20) { *why = "chunk_steps outside 1..2^20"; return KR_ERR_INVALID; }
  if (d->obs_ring < 0 || d->obs_ring > 4096) { *why = "obs_ring outside 0..4096"; return KR_ERR_INVALID; }
  if (d->max_slots < 0) { *why = "max_slots < 0"; return KR_ERR_INVALID; }
  if (d->n_maps < 1 || !d->rects || !d->map_rect_off) { *why = "need at least one map"; return KR_ERR_INVALID; }
  if (d->policy && d->net) { *why = "policy and net are exclusive (theta is one or the other)"; return KR_ERR_INVALID; }
  if (!(d->slice_ms >= 0 && d->slice_ms < 1e9)) { *why = "slice_ms outside [0, 1e9)"; return KR_ERR_INVALID; }
  return KR_OK;
}

int plan(const kr_server_desc *d, int32_t *capacity, uint64_t *per_slot, std::string *why) {
  int rc = check_desc(d, why);
  if (rc != KR_OK) return rc;
  const uint64_t ps = slot_bytes(*d), fx = fixed_bytes(*d);
  if (d->hbm_budget_bytes <= fx + 2 * ps) {
    *why = "HBM budget below the server's fixed " + std::to_string(fx) + " bytes plus two slots of " +
           std::to_string(ps) + " bytes";
    return KR_ERR_CAPACITY;
  }
  uint64_t cap = (d->hbm_budget_bytes - fx) / ps;
  if (d->max_slots > 0) cap = std::min<uint64_t>(cap, (uint64_t)d->max_slots);
  cap = std::min<uint64_t>(cap, 1u << 24);
  cap &= ~1ull;  // two equal partitions
  if (cap < 2) { *why = "fewer than two slots"; return KR_ERR_CAPACITY; }
  *capacity = (int32_t)cap;
  *per_slot = ps;
  return KR_OK;
}

template <typename T>
cudaError_t pinned_pair(T **h, T **d, size_t n) {
  cudaError_t e = cudaMallocHost(reinterpret_cast<void **>(h), std::max<size_t>(n, 1) * sizeof(T));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(d), std::max<size_t>(n, 1) * sizeof(T));
  return e;
}

void free_stage(Stage &s) {
  cudaFreeHost(s.h_pose); cudaFree(s.d_pose); cudaFreeHost(s.h_meta); cudaFree(s.d_meta);
  cudaFreeHost(s.h_slots); cudaFree(s.d_slots); cudaFreeHost(s.h_jobs); cudaFree(s.d_jobs);
  cudaFreeHost(s.h_theta); cudaFree(s.d_theta); cudaFreeHost(s.h_rslots); cudaFree(s.d_rslots);
  cudaFreeHost(s.h_res); cudaFree(s.d_res);
  s = Stage{};
}

// a request's results from its creatures' records (rec[0..population))
void complete(kr_server *S, Req &q, const SlotMeta *rec, double t) {
  const size_t n = q.slots.size();
  q.results.resize(n * KR_RESULT_WORDS);
  for (size_t i = 0; i < n; i++) slot_metrics(rec[i], q.results.data() + i * KR_RESULT_WORDS);
  q.completed = t;
  q.done = true;
  S->completed++;
  S->done_ids.push_back(q.id);
}

// completes the requests of partition p whose last round just ended (those
// completed while the slice ran have their results already) and frees
// their slots
void finish_round(kr_server *S, int p) {
  Round &R = S->round[p];
  const double t = S->now();
  if (R.timed) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, S->parts[p].ev0, S->parts[p].ev1) == cudaSuccess) S->device_ms += ms;
  }
  size_t off = 0;
  for (Req *qp : R.completing) {
    Req &q = *qp;
    const size_t n = q.slots.size();
    if (q.done) {
      S->done_unfreed -= (long)n;
    } else {
      complete(S, q, S->stage[p].h_res + off, t);
      off += n;
    }
    for (int s : q.slots) {
      S->b->h_meta[s].horizon = 0;
      S->b->h_remaining[s] = 0;
      S->free_slots.push_back(s);
      S->slot_req[s] = nullptr;
    }
    q.holding = false;
    S->part_used[p] -= (int)n;
  }
  if (!R.completing.empty()) {
    auto &act = S->active[p];
    act.erase(std::remove_if(act.begin(), act.end(), [](const Req *q) { return q->done; }), act.end());
    // the slot list keeps its order (admission order) without the freed slots
    auto &sl = S->parts[p].slots;
    sl.erase(std::remove_if(sl.begin(), sl.end(), [&](int s) { return S->b->h_meta[s].horizon == 0; }), sl.end());
    // requests released while their slice still held their slots
    for (const Req *q : R.completing)
      if (q->release_pending) S->reqs.erase(q->id);
  }
  R.completing.clear();
  R.inflight = false;
}

// admits arrived requests into free slots of partition p and stages them
int admit(kr_server *S, int p) {
  Stage &st = S->stage[p];
  cudaStream_t stream = S->streams[p];
  const double t = S->now();
  // the arrived requests that fit, in FIFO order
  AdmitScratch &A = S->adm;
  A.reqs.clear();
  int n_new = 0, n_theta = 0, theta_off = 0;
  {
    long free_left = (long)S->free_slots.size();
    int used = S->part_used[p];
    for (int64_t id : S->queue) {
      Req &q = S->reqs[id];
      if (q.arrival > t) break;
      const int pop = q.r.population;
      if (pop > free_left || used + pop > S->part_cap) break;
      if (!q.theta.empty()) {
        if (n_theta >= kMaxThetaPerRound) break;
        n_theta++;
      }
      free_left -= pop;
      used += pop;
      n_new += pop;
      A.reqs.push_back(&q);
    }
  }
  if (A.reqs.empty()) return KR_OK;
  // every admitted creature's initial data, one call, written into the staging
  A.arms.resize(n_new); A.segs.resize(n_new); A.maps.resize(n_new); A.hor.resize(n_new); A.ctrl.resize(n_new);
  A.xs.resize(n_new); A.ys.resize(n_new); A.an.resize(n_new); A.seeds.resize(n_new); A.tones.resize(n_new);
  int k = 0;
  for (const Req *qp : A.reqs) {
    const Req &q = *qp;
    const int pop = q.r.population;
    const int ctrl = q.theta.empty() ? KR_CTRL_STREAM : S->d.net ? KR_CTRL_NET : KR_CTRL_POLICY;
    for (int i = 0; i < pop; i++, k++) {
      A.arms[k] = q.r.arms; A.segs[k] = q.r.segs; A.maps[k] = q.r.map_id; A.hor[k] = q.r.horizon; A.ctrl[k] = ctrl;
      A.xs[k] = q.xs.empty() ? q.r.x : q.xs[i];
      A.ys[k] = q.xs.empty() ? q.r.y : q.ys[i];
      A.an[k] = q.xs.empty() ? q.r.angle : q.angles[i];
      A.seeds[k] = q.seeds.empty() ? (uint32_t)splitmix64(q.r.seed + (uint64_t)(q.r.first_individual + i)) : q.seeds[i];
      A.tones[k] = q.r.tone;
    }
  }
  int bad = -1;
  int rc = prepare_spawn_into(S->b, n_new, A.arms.data(), A.segs.data(), A.maps.data(), A.xs.data(), A.ys.data(),
                              A.an.data(), A.hor.data(), A.seeds.data(), A.tones.data(), KR_CTRL_STREAM, A.ctrl.data(),
                              st.h_pose, st.h_meta, &bad);
  if (rc != KR_OK) return S->batch_fail(rc);
  // slots, request tags, weight jobs and the host mirrors
  k = 0;
  for (Req *qp : A.reqs) {
    Req &q = *qp;
    const int pop = q.r.population;
    const bool pol = !q.theta.empty();
    q.slots.resize(pop);
    for (int i = 0; i < pop; i++) {
      const int s = S->free_slots.back();
      S->free_slots.pop_back();
      q.slots[i] = s;
    }
    for (int i = 0; i < pop; i++, k++) {
      const int s = q.slots[i];
      S->b->h_meta[s] = st.h_meta[k];
      S->b->h_remaining[s] = st.h_meta[k].horizon;
      st.h_meta[k].pad = q.slots[0];  // the request's tag: its first slot
      st.h_slots[k] = s;
      if (pol) {
        PJob &j = st.h_jobs[k];
        const int gi = q.r.first_individual + i;  // the individual's index in the whole population
        j.slot = s; j.theta_off = theta_off; j.arms = q.r.arms; j.segs = q.r.segs; j.pair = gi / 2;
        j.sign = (gi & 1) ? -1.f : 1.f; j.sigma = q.r.sigma; j.seed = q.r.seed;
        if (S->d.net) S->b->h_pw_arms[s] = q.r.arms;
        else S->b->h_pw_tpl[s] = st.h_meta[k].tpl;
      } else {
        st.h_jobs[k] = PJob{s, 0, 0, 0, 0, 1.f, 0.f, 0};
      }
    }
    if (pol) {
      std::copy(q.theta.begin(), q.theta.end(), st.h_theta + theta_off);
      theta_off += (int)q.theta.size();
    }
    if (S->d_done) S->prev_done[q.slots[0]] = 0;  // its count is cleared on the device below
    q.part = p;
    q.admitted = t;
    q.rounds_left = (q.r.horizon + S->chunk - 1) / S->chunk;
    q.pending = pop;
    q.seq = S->admitted;
    q.holding = true;
    S->part_used[p] += pop;
    S->active[p].push_back(&q);
    for (int s : q.slots) {
      S->parts[p].slots.push_back(s);
      S->slot_req[s] = &q;
    }
    S->queue.pop_front();
    S->admitted++;
  }
  if (n_new == 0) return KR_OK;
  cudaError_t e = cudaMemcpyAsync(st.d_pose, st.h_pose, (size_t)n_new * kStateStride * sizeof(float),
                                  cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st.d_meta, st.h_meta, (size_t)n_new * sizeof(SlotMeta), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(st.d_slots, st.h_slots, (size_t)n_new * sizeof(int), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = launch_spawn(S->b, st.d_slots, st.d_pose, st.d_meta, n_new, stream);
  if (e == cudaSuccess && S->d_done) {
    clear_done_kernel<<<(n_new + 255) / 256, 256, 0, stream>>>(st.d_meta, st.d_slots, n_new, S->d_done);
    e = cudaGetLastError();
  }
  const bool weights = S->d.policy || S->d.net;
  if (e == cudaSuccess && weights && theta_off > 0) {
    e = cudaMemcpyAsync(st.d_theta, st.h_theta, (size_t)theta_off * sizeof(float), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(st.d_jobs, st.h_jobs, (size_t)n_new * sizeof(PJob), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
      perturb_kernel<<<n_new, 256, 0, stream>>>(S->b->d_pw, weight_stride(S->d), st.d_theta, st.d_jobs, n_new,
                                                S->d.net);
      e = cudaGetLastError();
    }
  }
  if (e != cudaSuccess) return S->cuda_fail(e, "admission staging");
  S->h2d_bytes += (uint64_t)n_new * (kStateStride * sizeof(float) + sizeof(SlotMeta) + sizeof(int));
  if (weights && theta_off > 0) S->h2d_bytes += (uint64_t)theta_off * sizeof(float) + (uint64_t)n_new * sizeof(PJob);
  return KR_OK;
}

int run_round(kr_server *S, int p) {
  Round &R = S->round[p];
  if (R.inflight) {
    cudaError_t e = cudaEventSynchronize(R.done);
    if (e != cudaSuccess) return S->cuda_fail(e, "round wait");
    finish_round(S, p);
  }
  int rc = admit(S, p);
  if (rc != KR_OK) return rc;
  Part &P = S->parts[p];
  if (P.slots.empty()) return KR_OK;
  for (int s : P.slots) S->creature_steps += std::min(S->chunk, S->b->h_remaining[s]);
  P.dirty = true;
  rc = launch_part(S->b, P, S->chunk, true);
  if (rc != KR_OK) return S->batch_fail(rc);
  R.timed = true;
  // requests ending in this round: gather their results
  Stage &st = S->stage[p];
  int n_res = 0;
  for (Req *qp : S->active[p]) {
    Req &q = *qp;
    if (--q.rounds_left > 0) continue;
    R.completing.push_back(qp);
    for (int s : q.slots) st.h_rslots[n_res++] = s;
  }
  cudaStream_t stream = S->streams[p];
  cudaError_t e = cudaSuccess;
  if (n_res > 0) {
    e = cudaMemcpyAsync(st.d_rslots, st.h_rslots, (size_t)n_res * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
      gather_kernel<<<(n_res + 127) / 128, 128, 0, stream>>>(S->b->d_meta, st.d_rslots, n_res, st.d_res);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(st.h_res, st.d_res, (size_t)n_res * sizeof(SlotMeta), cudaMemcpyDeviceToHost, stream);
  }
  if (e == cudaSuccess) e = cudaEventRecord(R.done, stream);
  if (e != cudaSuccess) return S->cuda_fail(e, "round results");
  S->h2d_bytes += (uint64_t)n_res * sizeof(int);
  S->d2h_bytes += (uint64_t)n_res * sizeof(SlotMeta);
  R.inflight = true;
  S->rounds++;
  return KR_OK;
}

// Sliced scheduling.  After a slice: every slot's step counter from the
// device (the slice may have been cut short, so the host does not know how
// far each creature got), the requests whose creatures all reached their
// horizons gathered and completed (finish_round) unless that happened while
// the slice ran, their slots freed.
int finish_slice(kr_server *S) {
  Round &R = S->round[0];
  Part &P = S->parts[0];
  Stage &st = S->stage[0];
  cudaStream_t stream = S->streams[0];
  steps_kernel<<<(S->capacity + 255) / 256, 256, 0, stream>>>(S->b->d_meta, S->capacity, S->d_steps);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(S->h_steps, S->d_steps, (size_t)S->capacity * sizeof(int), cudaMemcpyDeviceToHost, stream);
  // the completion counts as the slice left them: the next slice's polls
  // count from here
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(S->h_done, S->d_done, (size_t)S->capacity * sizeof(int), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return S->cuda_fail(e, "slice step counters");
  S->d2h_bytes += 2 * (uint64_t)S->capacity * sizeof(int);
  std::copy(S->h_done, S->h_done + S->capacity, S->prev_done.begin());
  for (int s : P.slots) {
    SlotMeta &m = S->b->h_meta[s];
    const int done = std::min(S->h_steps[s], m.horizon);
    S->creature_steps += done - m.step;
    // a request ends with its last creature to reach its horizon
    if (done == m.horizon && m.step < m.horizon && --S->slot_req[s]->pending == 0)
      R.completing.push_back(S->slot_req[s]);
    m.step = done;
    S->b->h_remaining[s] = m.horizon - done;
  }
  std::sort(R.completing.begin(), R.completing.end(), [](const Req *a, const Req *b) { return a->seq < b->seq; });
  int n_res = 0;
  for (const Req *q : R.completing)
    if (!q->done)
      for (int s : q->slots) st.h_rslots[n_res++] = s;
  if (n_res > 0) {
    e = cudaMemcpyAsync(st.d_rslots, st.h_rslots, (size_t)n_res * sizeof(int), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) {
      gather_kernel<<<(n_res + 127) / 128, 128, 0, stream>>>(S->b->d_meta, st.d_rslots, n_res, st.d_res);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(st.h_res, st.d_res, (size_t)n_res * sizeof(SlotMeta), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return S->cuda_fail(e, "slice results");
    S->h2d_bytes += (uint64_t)n_res * sizeof(int);
    S->d2h_bytes += (uint64_t)n_res * sizeof(SlotMeta);
  }
  finish_round(S, 0);
  return KR_OK;
}

// While a slice runs: the device's per-request completion counts, copied
// back at most once every kPollS seconds; the requests whose creatures all
// reached their horizons since the poll before are completed at once --
// their records copied back by the copy engine while the kernel goes on
// (the kernel writes a creature's record before counting it).  Their slots
// return to the pool when the slice ends.
constexpr double kPollS = 1e-3;

int poll_completions(kr_server *S) {
  const double t = S->now();
  if (!S->round[0].inflight || t - S->polled < kPollS) return KR_OK;
  S->polled = t;
  cudaError_t e = cudaMemcpyAsync(S->h_done, S->d_done, (size_t)S->capacity * sizeof(int), cudaMemcpyDeviceToHost,
                                  S->ctl);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S->ctl);
  if (e != cudaSuccess) return S->cuda_fail(e, "completion counts");
  S->d2h_bytes += (uint64_t)S->capacity * sizeof(int);
  std::vector<Req *> ended;
  for (int tag = 0; tag < S->capacity; tag++) {
    if (S->h_done[tag] == S->prev_done[tag]) continue;
    S->prev_done[tag] = S->h_done[tag];
    Req *q = S->slot_req[tag];
    if (q && !q->done && q->slots[0] == tag && S->h_done[tag] >= (int)q->slots.size()) ended.push_back(q);
  }
  if (ended.empty()) return KR_OK;
  std::sort(ended.begin(), ended.end(), [](const Req *a, const Req *b) { return a->seq < b->seq; });
  // the records, read by the copy engine (the running slice holds every SM):
  // runs of nearby slots, one copy each, into the slice's result staging,
  // which is idle until the slice ends (runs are disjoint ranges of the
  // slots, so they fit its capacity records)
  Stage &st = S->stage[0];
  std::vector<int> &want = S->gather_slots;
  want.clear();
  for (const Req *q : ended) want.insert(want.end(), q->slots.begin(), q->slots.end());
  std::sort(want.begin(), want.end());
  constexpr int kRunGap = 16;  // records copied across a gap rather than a copy more
  size_t off = 0;
  for (size_t i = 0; i < want.size() && e == cudaSuccess;) {
    const int a = want[i];
    int b = a;
    size_t j = i + 1;
    while (j < want.size() && want[j] - b <= kRunGap) b = want[j++];
    e = cudaMemcpyAsync(st.h_res + off, S->b->d_meta + a, (size_t)(b - a + 1) * sizeof(SlotMeta),
                        cudaMemcpyDeviceToHost, S->ctl);
    for (size_t k = i; k < j; k++) S->rec_pos[want[k]] = (int)(off + (size_t)(want[k] - a));
    off += (size_t)(b - a + 1);
    i = j;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(S->ctl);
  if (e != cudaSuccess) return S->cuda_fail(e, "streamed results");
  S->d2h_bytes += (uint64_t)off * sizeof(SlotMeta);
  const double tc = S->now();
  std::vector<SlotMeta> rec;
  for (Req *q : ended) {
    rec.resize(q->slots.size());
    for (size_t i = 0; i < q->slots.size(); i++) rec[i] = st.h_res[S->rec_pos[q->slots[i]]];
    complete(S, *q, rec.data(), tc);
    S->done_unfreed += (long)q->slots.size();
  }
  return KR_OK;
}

// true when the queue's first request has arrived and fits the free slots
// plus those of the requests completed while the slice runs
bool admissible(kr_server *S) {
  if (S->queue.empty()) return false;
  const Req &q = S->reqs.at(S->queue.front());
  const double t = S->now();
  if (q.arrival > t) return false;
  // a slice runs at least 10 host gaps before an admission cuts it, so that
  // the GPU idles at most about a tenth of the time however often requests
  // come (with 3, queued single-creature requests cut slices so often that
  // the host gaps took 8 % of a 65k memory-bound run)
  if (S->round[0].inflight && t - S->slice_t0 < 10 * S->gap_s) return false;
  return q.r.population <= (long)S->free_slots.size() + S->done_unfreed;
}

// One step of sliced scheduling: while a slice runs, complete the requests
// it has finished (poll_completions) and preempt it if an arrived request
// fits or its time is up (otherwise return at once); after it, free the
// completed requests' slots, admit and launch the next slice, every live
// creature up to its horizon (at most chunk_steps env steps).  A relaunch
// regroups the creatures by their remaining steps and spreads the longest
// over every SM, so that the tail of long horizons runs with short steps:
// slices make the rollouts' device time shorter, not only admissions sooner.
int run_slice(kr_server *S) {
  Round &R = S->round[0];
  cudaError_t e;
  if (R.inflight && !S->stop_sent) {
    int rc = poll_completions(S);
    if (rc != KR_OK) return rc;
    // the time slice: slice_ms, or 10 host gaps when those are longer (large
    // populations), so that the GPU idles at most about a tenth of the time
    const bool time_up = S->now() - S->slice_t0 >= std::max(S->slice_s, 10 * S->gap_s);
    if (!admissible(S) && !time_up) {
      e = cudaEventQuery(R.done);
      if (e == cudaErrorNotReady) return KR_OK;
      if (e != cudaSuccess) return S->cuda_fail(e, "slice query");
    } else {
      e = cudaMemcpyAsync(S->d_stop, S->h_flag + 1, sizeof(int), cudaMemcpyHostToDevice, S->ctl);
      if (e != cudaSuccess) return S->cuda_fail(e, "slice stop");
      S->stop_sent = true;
    }
  }
  double ended = -1;
  if (R.inflight) {
    e = cudaEventSynchronize(R.done);
    // the stop word's copy has landed before the next slice clears it
    if (e == cudaSuccess && S->stop_sent) e = cudaStreamSynchronize(S->ctl);
    if (e != cudaSuccess) return S->cuda_fail(e, "slice wait");
    ended = S->now();
    int rc = finish_slice(S);
    if (rc != KR_OK) return rc;
  }
  int rc = admit(S, 0);
  if (rc != KR_OK) return rc;
  Part &P = S->parts[0];
  if (P.slots.empty()) return KR_OK;
  cudaStream_t stream = S->streams[0];
  e = cudaMemcpyAsync(S->d_stop, S->h_flag, sizeof(int), cudaMemcpyHostToDevice, stream);
  // the slice's copies of the completion counts follow its admissions' resets
  if (e == cudaSuccess) e = cudaEventRecord(S->staged, stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(S->ctl, S->staged, 0);
  if (e != cudaSuccess) return S->cuda_fail(e, "slice start");
  P.dirty = true;
  rc = launch_part(S->b, P, S->chunk, true);
  if (rc != KR_OK) return S->batch_fail(rc);
  R.timed = true;
  e = cudaEventRecord(R.done, stream);
  if (e != cudaSuccess) return S->cuda_fail(e, "slice record");
  R.inflight = true;
  S->stop_sent = false;
  S->slice_t0 = S->now();
  if (ended >= 0) {
    const double gap = S->slice_t0 - ended;
    S->gap_s = S->gap_s > 0 ? 0.75 * S->gap_s + 0.25 * gap : gap;
    S->gap_sum += gap;
  }
  S->rounds++;
  return KR_OK;
}

bool busy(const kr_server *S) {
  return !S->queue.empty() || !S->active[0].empty() || !S->active[1].empty() || S->round[0].inflight ||
         S->round[1].inflight;
}

}  // namespace

extern "C" int kr_server_plan(const kr_server_desc *d, int32_t *capacity, uint64_t *bytes_per_slot) {
  int32_t cap = 0;
  uint64_t ps = 0;
  int rc = plan(d, &cap, &ps, &g_serve_error);
  if (rc != KR_OK) return rc;
  if (capacity) *capacity = cap;
  if (bytes_per_slot) *bytes_per_slot = ps;
  return KR_OK;
}

extern "C" int kr_server_create(const kr_server_desc *d, kr_server **out) {
  if (!out) { g_serve_error = "null output"; return KR_ERR_INVALID; }
  *out = nullptr;
  int32_t cap = 0;
  uint64_t ps = 0;
  int rc = plan(d, &cap, &ps, &g_serve_error);
  if (rc != KR_OK) return rc;
  kr_batch_desc bd{};
  bd.solver = d->solver;
  bd.n_maps = d->n_maps;
  bd.rects = d->rects;
  bd.map_rect_off = d->map_rect_off;
  bd.capacity = cap;
  bd.obs_ring = d->obs_ring;
  bd.grip_slip_max = d->grip_slip_max;
  bd.grip_cooldown = d->grip_cooldown;
  bd.control_mode = d->net ? KR_CTRL_NET : KR_CTRL_STREAM;  // per slot: policy / net for requests with theta
  bd.control_period = 6;
  if (d->net) {
    bd.lights = d->lights;
    bd.map_light_off = d->map_light_off;
    bd.map_size = d->map_size;
  }
  kr_batch *b = nullptr;
  rc = kr_batch_create(&bd, &b);
  if (rc != KR_OK) { g_serve_error = std::string("engine: ") + kr_batch_last_error(nullptr); return rc; }
  kr_server *S = new kr_server();
  S->d = *d;
  S->d.rects = nullptr;
  S->d.map_rect_off = nullptr;
  S->d.lights = nullptr;
  S->d.map_light_off = nullptr;
  S->d.map_size = nullptr;
  S->b = b;
  S->capacity = cap;
  S->sliced = d->slice_ms > 0;
  S->slice_s = d->slice_ms * 1e-3;
  S->part_cap = S->sliced ? cap : cap / 2;
  S->chunk = d->chunk_steps;
  S->bytes_per_slot = ps;
  S->t0 = std::chrono::steady_clock::now();
  auto bail = [&](int code) {
    g_serve_error = S->err;
    kr_server_destroy(S);
    return code;
  };
  if (d->lanes_per_creature > 0 || d->warps_per_cta > 0 || d->ctas_per_sm > 0) {
    rc = kr_batch_set_launch(b, d->lanes_per_creature > 0 ? d->lanes_per_creature : 16,
                             d->warps_per_cta > 0 ? d->warps_per_cta : 8, std::max(0, d->ctas_per_sm));
    if (rc != KR_OK) { S->batch_fail(rc); return bail(rc); }
  }
  // every body shape up front: no template upload while rounds are in flight
  for (int a = 1; a <= KR_BATCH_MAX_ARMS; a++)
    for (int sg = 1; sg <= KR_BATCH_MAX_SEGS; sg++)
      if (ensure_template(b, a, sg) < 0) { S->err = "template build failed"; return bail(KR_ERR_INVALID); }
  rc = upload_templates(b);
  if (rc == KR_OK) rc = plan_shape(b);
  if (rc != KR_OK) { S->batch_fail(rc); return bail(rc); }
  cudaError_t e = cudaSuccess;
  if (d->policy || d->net) {
    const int ws = weight_stride(*d);  // a multiple of 4: 16-byte aligned individuals
    e = cudaMalloc(&b->d_pw, (size_t)cap * ws * sizeof(float));
    std::vector<int> idx(cap);
    for (int s = 0; s < cap; s++) idx[s] = s;
    if (e == cudaSuccess) e = cudaMalloc(&b->d_pw_idx, (size_t)cap * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(b->d_pw_idx, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->d_pw, 0, (size_t)cap * ws * sizeof(float));
    b->pw_stride = ws;
    b->pw_capacity = (size_t)cap * ws;
    b->n_individuals = cap;
    b->h_pw_idx = idx;
    b->h_pw_tpl.assign(cap, -1);
    b->h_pw_arms.assign(cap, -1);
    if (e != cudaSuccess) { S->cuda_fail(e, "policy weights"); return bail(KR_ERR_CUDA); }
  }
  if (S->sliced) {
    if (e == cudaSuccess) e = cudaMalloc(&S->d_stop, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(S->d_stop, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_flag, 2 * sizeof(int));
    if (e == cudaSuccess) { S->h_flag[0] = 0; S->h_flag[1] = 1; }
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_steps, (size_t)cap * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&S->d_steps, (size_t)cap * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&S->d_done, (size_t)cap * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(S->d_done, 0, (size_t)cap * sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&S->h_done, (size_t)cap * sizeof(int));
    S->parts[0].tag_done = S->d_done;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->ctl, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->staged, cudaEventDisableTiming);
    S->prev_done.assign(cap, 0);
    S->rec_pos.assign(cap, 0);
    S->parts[0].stop = S->d_stop;
  }
  for (int p = 0; p < (S->sliced ? 1 : 2); p++) {
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->streams[p], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&S->round[p].done, cudaEventDisableTiming);
    S->parts[p].all = false;
    S->parts[p].stream = S->streams[p];
    Stage &st = S->stage[p];
    const size_t pc = (size_t)S->part_cap;
    if (e == cudaSuccess) e = pinned_pair(&st.h_pose, &st.d_pose, pc * kStateStride);
    if (e == cudaSuccess) e = pinned_pair(&st.h_meta, &st.d_meta, pc);
    if (e == cudaSuccess) e = pinned_pair(&st.h_slots, &st.d_slots, pc);
    if (e == cudaSuccess) e = pinned_pair(&st.h_jobs, &st.d_jobs, pc);
    if (e == cudaSuccess)
      e = pinned_pair(&st.h_theta, &st.d_theta,
                      d->policy || d->net ? (size_t)kMaxThetaPerRound * weight_stride(*d) : 1);
    if (e == cudaSuccess) e = pinned_pair(&st.h_rslots, &st.d_rslots, pc);
    if (e == cudaSuccess) e = pinned_pair(&st.h_res, &st.d_res, pc);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { S->cuda_fail(e, "server setup"); return bail(KR_ERR_CUDA); }
  S->free_slots.resize(cap);
  for (int s = 0; s < cap; s++) S->free_slots[s] = cap - 1 - s;  // lowest slots first
  S->slot_req.assign(cap, nullptr);
  S->device_bytes = ps * (uint64_t)cap + fixed_bytes(*d);
  *out = S;
  return KR_OK;
}

extern "C" double kr_server_now(const kr_server *s) { return s ? s->now() : 0.0; }

extern "C" int kr_server_submit(kr_server *S, const kr_request *r, int64_t *id) {
  if (!S || !r) return KR_ERR_INVALID;
  if (r->population < 1 || r->population > S->part_cap)
    return S->fail(KR_ERR_CAPACITY, "population " + std::to_string(r->population) + " outside 1.." +
                                        std::to_string(S->part_cap) + (S->sliced ? " (the slots)" : " (half the slots)"));
  if (r->horizon < 1) return S->fail(KR_ERR_INVALID, "horizon < 1");
  if (r->first_individual < 0 || (r->first_individual & 1))
    return S->fail(KR_ERR_INVALID, "first_individual must be even and >= 0");
  if (r->arms < 1 || r->arms > KR_BATCH_MAX_ARMS || r->segs < 1 || r->segs > KR_BATCH_MAX_SEGS)
    return S->fail(KR_ERR_INVALID, "body shape outside 1..8 arms x 1..9 segments");
  if (r->map_id < 0 || r->map_id >= S->d.n_maps) return S->fail(KR_ERR_INDEX, "unknown map");
  if (!r->xs && !(std::isfinite(r->x) && std::isfinite(r->y) && std::isfinite(r->angle)))
    return S->fail(KR_ERR_INVALID, "spawn pose not finite");
  Req q;
  q.id = S->next_id++;
  q.r = *r;
  q.r.theta = nullptr;
  if (r->theta) {
    if (!S->d.policy && !S->d.net) return S->fail(KR_ERR_STATE, "server created without policy or net weights");
    const int need = S->d.net ? net_param_count(r->arms) : policy_param_count(r->arms, r->segs);
    if (r->n_params < need)
      return S->fail(KR_ERR_INVALID, "theta has " + std::to_string(r->n_params) + " parameters, a " +
                                         std::to_string(r->arms) + "x" + std::to_string(r->segs) + " body needs " +
                                         std::to_string(need));
    if (!(std::isfinite(r->sigma))) return S->fail(KR_ERR_INVALID, "sigma not finite");
    q.theta.assign(r->theta, r->theta + need);
  }
  const bool px = r->xs != nullptr, py = r->ys != nullptr, pa = r->angles != nullptr;
  if (px != py || px != pa) return S->fail(KR_ERR_INVALID, "per-individual poses need xs, ys and angles");
  if (px) {
    q.xs.assign(r->xs, r->xs + r->population);
    q.ys.assign(r->ys, r->ys + r->population);
    q.angles.assign(r->angles, r->angles + r->population);
    for (int i = 0; i < r->population; i++)
      if (!(std::isfinite(q.xs[i]) && std::isfinite(q.ys[i]) && std::isfinite(q.angles[i])))
        return S->fail(KR_ERR_INVALID, "spawn pose not finite");
  }
  if (r->control_seeds) q.seeds.assign(r->control_seeds, r->control_seeds + r->population);
  q.r.xs = q.r.ys = q.r.angles = nullptr;
  q.r.control_seeds = nullptr;
  q.arrival = r->arrival < 0 ? S->now() : r->arrival;
  // FIFO by arrival time (requests submitted ahead of their arrival keep their order)
  auto it = S->queue.end();
  while (it != S->queue.begin() && S->reqs[*(it - 1)].arrival > q.arrival) --it;
  S->queue.insert(it, q.id);
  S->reqs.emplace(q.id, std::move(q));
  S->submitted++;
  if (id) *id = S->next_id - 1;
  return KR_OK;
}

extern "C" int kr_server_submit_batch(kr_server *S, const kr_request *reqs, int32_t n, int64_t *ids,
                                      int32_t *n_submitted) {
  if (!S || (n > 0 && !reqs)) return KR_ERR_INVALID;
  int k = 0, rc = KR_OK;
  for (; k < n; k++) {
    int64_t id = 0;
    rc = kr_server_submit(S, reqs + k, &id);
    if (rc != KR_OK) break;
    if (ids) ids[k] = id;
  }
  if (n_submitted) *n_submitted = k;
  return rc;
}

extern "C" int kr_server_pump(kr_server *S, int32_t *busy_out) {
  if (!S) return KR_ERR_INVALID;
  int rc;
  if (S->sliced) {
    rc = run_slice(S);
  } else {
    const int p = S->next;
    S->next ^= 1;
    rc = run_round(S, p);
  }
  if (busy_out) *busy_out = busy(S) ? 1 : 0;
  return rc;
}

extern "C" int kr_server_drain(kr_server *S) {
  if (!S) return KR_ERR_INVALID;
  while (busy(S)) {
    if (!S->round[0].inflight && !S->round[1].inflight && S->active[0].empty() && S->active[1].empty() &&
        !S->queue.empty()) {
      const double wait = S->reqs[S->queue.front()].arrival - S->now();
      if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 1.0)));
    }
    int rc = kr_server_pump(S, nullptr);
    if (rc != KR_OK) return rc;
    // a slice that runs on with nothing to preempt it: look again shortly
    if (S->sliced && S->round[0].inflight && !S->stop_sent)
      std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  return KR_OK;
}

extern "C" int kr_server_poll(kr_server *S, int64_t *ids, int32_t cap, int32_t *n) {
  if (!S || !n || (cap > 0 && !ids)) return KR_ERR_INVALID;
  const int k = std::min<int>(cap, (int)S->done_ids.size());
  for (int i = 0; i < k; i++) ids[i] = S->done_ids[i];
  S->done_ids.erase(S->done_ids.begin(), S->done_ids.begin() + k);
  *n = k;
  return KR_OK;
}

namespace {
// the request `id` as the caller sees it (a released request is gone)
Req *find_req(kr_server *S, int64_t id) {
  auto it = S->reqs.find(id);
  return it == S->reqs.end() || it->second.release_pending ? nullptr : &it->second;
}

// releases a completed request: erased at once or, while the slice that
// completed it still holds its slots, when the slice frees them
void release_req(kr_server *S, Req &q) {
  if (q.holding) q.release_pending = true;
  else S->reqs.erase(q.id);
}
}  // namespace

extern "C" int kr_server_result(kr_server *S, int64_t id, double *results, double *times) {
  if (!S) return KR_ERR_INVALID;
  const Req *qp = find_req(S, id);
  if (!qp) return S->fail(KR_ERR_INDEX, "unknown request " + std::to_string(id));
  const Req &q = *qp;
  if (!q.done) return S->fail(KR_ERR_STATE, "request " + std::to_string(id) + " has not completed");
  if (results) std::copy(q.results.begin(), q.results.end(), results);
  if (times) { times[0] = q.arrival; times[1] = q.admitted; times[2] = q.completed; }
  return KR_OK;
}

extern "C" int kr_server_result_batch(kr_server *S, const int64_t *ids, int32_t n, double *results,
                                      double *times, int32_t release) {
  if (!S || (n > 0 && !ids)) return KR_ERR_INVALID;
  for (int k = 0; k < n; k++) {
    const Req *q = find_req(S, ids[k]);
    if (!q) return S->fail(KR_ERR_INDEX, "unknown request " + std::to_string(ids[k]));
    if (!q->done) return S->fail(KR_ERR_STATE, "request " + std::to_string(ids[k]) + " has not completed");
  }
  size_t off = 0;
  for (int k = 0; k < n; k++) {
    Req *q = find_req(S, ids[k]);
    if (!q) return S->fail(KR_ERR_INDEX, "request " + std::to_string(ids[k]) + " listed twice after its release");
    if (results) std::copy(q->results.begin(), q->results.end(), results + off);
    off += q->results.size();
    if (times) { times[3 * k] = q->arrival; times[3 * k + 1] = q->admitted; times[3 * k + 2] = q->completed; }
    if (release) release_req(S, *q);
  }
  return KR_OK;
}

extern "C" int kr_server_release(kr_server *S, int64_t id) {
  if (!S) return KR_ERR_INVALID;
  Req *q = find_req(S, id);
  if (!q) return S->fail(KR_ERR_INDEX, "unknown request " + std::to_string(id));
  if (!q->done) return S->fail(KR_ERR_STATE, "request " + std::to_string(id) + " has not completed");
  release_req(S, *q);
  return KR_OK;
}

extern "C" int kr_server_get_stats(kr_server *S, kr_server_stats *o) {
  if (!S || !o) return KR_ERR_INVALID;
  o->capacity = S->capacity;
  o->partition_capacity = S->part_cap;
  o->live = S->part_used[0] + S->part_used[1];
  o->queued = (int32_t)S->queue.size();
  o->submitted = S->submitted;
  o->admitted = S->admitted;
  o->completed = S->completed;
  o->rounds = S->rounds;
  o->creature_steps = S->creature_steps;
  o->device_ms = S->device_ms;
  o->bytes_per_slot = S->bytes_per_slot;
  o->device_bytes = S->device_bytes;
  o->h2d_bytes = S->h2d_bytes + S->parts[0].h2d_bytes + S->parts[1].h2d_bytes;
  o->d2h_bytes = S->d2h_bytes;
  o->host_gap_ms = S->gap_sum * 1e3;
  return KR_OK;
}

extern "C" int kr_policy_eps(uint64_t seed, int32_t pair, int32_t n, float *out) {
  if (!out || n < 0) { g_serve_error = "kr_policy_eps: bad arguments"; return KR_ERR_INVALID; }
  if (n == 0) return KR_OK;
  float *d = nullptr;
  cudaError_t e = cudaMalloc(&d, (size_t)n * sizeof(float));
  if (e == cudaSuccess) {
    eps_kernel<<<(n + 255) / 256, 256>>>(seed, pair, n, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  if (d) cudaFree(d);
  if (e != cudaSuccess) { g_serve_error = cudaGetErrorString(e); return KR_ERR_CUDA; }
  return KR_OK;
}

extern "C" void kr_server_destroy(kr_server *S) {
  if (!S) return;
  // a running slice stops at its creatures' next env step instead of running
  // them to their horizons
  if (S->sliced && S->round[0].inflight && !S->stop_sent)
    cudaMemcpyAsync(S->d_stop, S->h_flag + 1, sizeof(int), cudaMemcpyHostToDevice, S->ctl);
  cudaDeviceSynchronize();
  for (int p = 0; p < 2; p++) {
    free_part(S->parts[p]);
    free_stage(S->stage[p]);
    if (S->round[p].done) cudaEventDestroy(S->round[p].done);
    if (S->streams[p]) cudaStreamDestroy(S->streams[p]);
  }
  if (S->d_stop) cudaFree(S->d_stop);
  if (S->h_flag) cudaFreeHost(S->h_flag);
  if (S->h_steps) cudaFreeHost(S->h_steps);
  if (S->d_steps) cudaFree(S->d_steps);
  if (S->d_done) cudaFree(S->d_done);
  if (S->h_done) cudaFreeHost(S->h_done);
  if (S->ctl) cudaStreamDestroy(S->ctl);
  if (S->staged) cudaEventDestroy(S->staged);
  if (S->b) kr_batch_destroy(S->b);
  delete S;
}

extern "C" const char *kr_server_last_error(const kr_server *S) {
  return S ? S->err.c_str() : g_serve_error.c_str();
}
