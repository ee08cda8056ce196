/*
 * kraken_b200.h -- C ABI of the B200 (sm_100a) XPBD creature-step library.
 *
 * Drop-in boundary for Kraken 3's src/gpu/gpuworld.js.  Each entry point
 * names the reference function it replaces (file:line in the reference
 * project).  Plain pointers and sizes only; every call returns an int status
 * (KR_OK == 0) and never throws; host pointers are borrowed for the duration
 * of the call.  A handle is not thread-safe: one host thread and one CUDA
 * stream per handle, like the reference's single JS thread per device.
 *
 * Buffer layouts are the reference's (gpuworld.js:12-19, solver.wgsl:37-54):
 *   body        12 x f32 = 48 B   px py ppx ppy vx vy ang angP av invMass invInertia pad
 *   constraint  20 x u32 = 80 B   aIdx bIdx cType owner | lax lay lbx lby |
 *                                 compliance rest target minAng | maxAng lamX lamY lam |
 *                                 breakForce broken pad pad   (u32 words: 0-3, 17-19)
 *   collPt       4 x u32 = 16 B   body(u32) lx ly r
 *   rect         4 x f32 = 16 B   x y w h
 *   force        4 x f32 = 16 B   fx fy torque adhesion
 * so that mirrorInto / packControls (gpuworld.js:331-456) stay bit-exact on
 * the caller's side.
 */
#ifndef KRAKEN_B200_H
#define KRAKEN_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define KR_OK 0
#define KR_ERR_INVALID 1   /* implausible parameter (gpuworld.js:224-229)            */
#define KR_ERR_INDEX 2     /* body index out of range (gpuworld.js:269-271)          */
#define KR_ERR_CUDA 3      /* CUDA runtime error; the message says which call         */
#define KR_ERR_CAPACITY 4  /* a connected component is larger than the kernel holds  */
#define KR_ERR_STATE 5     /* call order: step/download before upload                 */
#define KR_ERR_NODEVICE 6  /* no CUDA device (isAvailable, gpuworld.js:30-32)         */

#define KR_BODY_WORDS 12
#define KR_CONS_WORDS 20
#define KR_COLLPT_WORDS 4
#define KR_RECT_WORDS 4
#define KR_FORCE_WORDS 4

/* island capacity of the step kernel (one creature per warp) */
#define KR_MAX_ISLAND_BODIES 160
#define KR_MAX_ISLAND_CONSTRAINTS 384
#define KR_MAX_ISLAND_COLLPTS 384
#define KR_MAX_LEVELS 96

typedef struct kr_world kr_world;

/* Solver constants as the CPU world holds them (XpbdWorld, xpbd.js:189-197).
 * The f32 copies the kernel uses are derived exactly as writeStatic
 * (gpuworld.js:209-223) and f32solver.mjs:79-85 derive them. */
typedef struct kr_solver_params {
  double h;             /* s per substep, 0 < h < 1 */
  int32_t substeps;     /* >= 1 */
  int32_t iterations;   /* 1..64 */
  double lin_drag;      /* 1/s */
  double ang_drag;      /* 1/s */
  double max_speed;     /* px/s */
  double max_ang_speed; /* rad/s */
} kr_solver_params;

/* isAvailable (gpuworld.js:30-32): number of CUDA devices, 0 if none. */
int kr_device_count(void);

/* create + writeStatic (gpuworld.js:34-171, 209-247).
 *   rects      n_rects x 4 f32 (map.rects as the reference's rectData)
 *   coll_pts   n_coll_pts x 4 words in groupCollPoints order (gpuworld.js:189-207)
 *   coll_range 2 x n_bodies u32: [offset(0..n-1), count(0..n-1)]
 * Validates exactly the reference's sanity guards and returns
 * KR_ERR_INVALID with a message for an implausible value. */
int kr_create(const kr_solver_params *params, uint32_t n_bodies, uint32_t n_constraints,
              const float *rects, uint32_t n_rects, const uint32_t *coll_pts,
              uint32_t n_coll_pts, const uint32_t *coll_range, kr_world **out);

/* upload (gpuworld.js:250-298): full CPU->device state.
 *   bodies     n_bodies x 12 f32
 *   cons       n_constraints x 20 words, in solve (colour-grouped) order
 *   forces     n_bodies x 4 f32, may be NULL (all zero)
 *   color_info 33 u32 [off(16), cnt(16), workgroups], may be NULL; when given
 *              the 16 ranges must tile [0, n_constraints) in order.
 * Re-derives the per-creature solve schedule from the constraint topology.
 * KR_ERR_INDEX if a body index is out of range. */
int kr_upload(kr_world *w, const float *bodies, const uint32_t *cons, const float *forces,
              const uint32_t *color_info);

/* uploadControls (gpuworld.js:312-315): takes only the control fields of the
 * 80 B records (lbx o+6, lby o+7, compliance o+8, target o+10,
 * breakForce o+16, broken o+17 as u32), exactly what packControls writes. */
int kr_upload_controls(kr_world *w, const uint32_t *cons);

/* step (gpuworld.js:374-382) repeated n_steps times: substeps x (resetLambda,
 * integrate, iterations x (colour sweep, collisions), finalize) + gripBreak.
 * Asynchronous on the handle's stream. */
int kr_step(kr_world *w, int32_t n_steps);

/* download (gpuworld.js:385-396) without the mirror: copies the device state
 * back into the caller's 48 B / 80 B blocks (either may be NULL). Synchronous. */
int kr_download(kr_world *w, float *bodies, uint32_t *cons);

/* Block until the handle's queued work has finished. */
int kr_sync(kr_world *w);

/* Use an existing CUDA stream (cudaStream_t passed as void*; NULL = the
 * handle's own stream). */
int kr_set_stream(kr_world *w, void *stream);

/* Number of connected components (creatures) the last upload found, and the
 * number of constraint levels of the largest one. */
int kr_world_islands(const kr_world *w, int32_t *n_islands, int32_t *max_levels);

/* Allocation-free step.  No counterpart in the reference: gpuworld.js always
 * owns its device buffers.  This entry point is for callers that cannot
 * allocate GPU memory themselves or through this library -- code inside a
 * host application's own device-memory pool, an embedding that must own
 * every allocation, or a latency-critical loop where a cudaMalloc (and the
 * synchronization it implies) is not allowed.  It advances the world n_steps
 * env steps exactly like kr_step (same kernel, same results), with every
 * buffer in device memory owned by the caller:
 *   bodies   n_bodies x 12 f32 (in/out)     cons   n_constraints x 20 words (in/out)
 *   forces   n_bodies x 4 f32 (in/out)      rects  n_rects x 4 f32 (x y w h)
 *   coll_pts n_coll_pts x 4 words and coll_range 2 x n_bodies u32, as for kr_create.
 * Alignment: bodies, forces, cons and coll_pts must start on a 16-byte
 * boundary (the kernel moves them as 16-byte vectors), rects and coll_range
 * on a 4-byte one; a misaligned pointer is rejected with KR_ERR_INVALID
 * before the device is touched.
 * The per-creature schedule is rebuilt on the device at every call into one
 * file-scope device array of fixed size (about 270 KB; every GPU that loads
 * the library holds it until the process exits), so the call allocates
 * nothing, neither on the device nor on the host.  Limits: at most
 * KR_NOALLOC_MAX_BODIES bodies, KR_NOALLOC_MAX_CONSTRAINTS constraints,
 * KR_NOALLOC_MAX_COLLPTS collision points and KR_NOALLOC_MAX_RECTS rects;
 * larger worlds are rejected with KR_ERR_CAPACITY before any GPU work, and a
 * creature above the KR_MAX_ISLAND_* capacities is found by the schedule
 * builder and rejected with the same code before any step runs.  Other codes: KR_ERR_INVALID
 * (null pointer, implausible parameter, inconsistent coll_range),
 * KR_ERR_INDEX (a constraint's body index out of range), KR_ERR_CUDA.  No
 * message is recorded (recording one would allocate).  A rejected world
 * leaves the caller's buffers untouched.
 * The first call on a device looks up the device address of the scratch
 * array.  Every call waits on the host for the schedule builder's verdict --
 * a 4-byte copy from the device into static host memory followed by a
 * synchronize of `stream` (cudaStream_t as void*, NULL = the legacy default
 * stream) -- and only then enqueues the steps asynchronously; so no call can
 * be made inside a stream capture (the copy and the synchronize are not
 * capturable, and the capture would be invalidated).  Every call on a
 * device shares the one scratch array: calls that overlap on the GPU (other
 * host threads, other streams) race and must not be issued. */
#define KR_NOALLOC_MAX_BODIES 2048
#define KR_NOALLOC_MAX_CONSTRAINTS 4096
#define KR_NOALLOC_MAX_COLLPTS 4096
#define KR_NOALLOC_MAX_RECTS 1024
int kr_step_noalloc(const kr_solver_params *params, uint32_t n_bodies, uint32_t n_constraints,
                    float *bodies, uint32_t *cons, float *forces, const float *rects,
                    uint32_t n_rects, const uint32_t *coll_pts, uint32_t n_coll_pts,
                    const uint32_t *coll_range, int32_t n_steps, void *stream);

/* destroy (gpuworld.js:466-472): frees device memory; NULL is a no-op. */
void kr_destroy(kr_world *w);

/* Message of the last failing call on this handle, or of the last failing
 * kr_create / kr_device_count when w is NULL. Never NULL. */
const char *kr_last_error(const kr_world *w);

#ifdef __cplusplus
}
#endif
#endif
