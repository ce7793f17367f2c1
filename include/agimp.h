/*
 * agimp.h -- C ABI of the B200 adaptive GIMP substep library (libagimp.so).
 *
 * The reference project (g1n0st/adaptive-gimp) exposes this path as the Python
 * class AdaptiveGIMP (adaptive_gimp.py:4-352).  Each entry point below names
 * the part of that interface it replaces.  The Python facade in
 * adaptive-gimp_b200/agimp/simulator.py binds these functions with ctypes and
 * mirrors the reference's constructor, fields and substep().
 *
 * Conventions
 *  - Plain pointers and sizes only.  `stream` is a cudaStream_t (NULL = legacy
 *    default stream).  Every call is ordered on `stream`; calls that return
 *    data into HOST memory synchronize `stream` before returning.
 *  - `memory` says where caller buffers live: AGIMP_MEM_DEVICE (device
 *    pointers on the simulator's device) or AGIMP_MEM_HOST (host pointers,
 *    pinned or pageable).
 *  - Particle arrays use the reference's field layout (Taichi to_numpy):
 *    vectors [N][dim], matrices [N][dim][dim] row-major, f32.
 *  - Grid readback is a dense box of indices [lo, lo+n) per axis, first axis
 *    slowest (the reference's ti.ij / ti.ijk order).  The library stores every
 *    level over indices [-4, size+8); readback outside reads 0.
 *  - The library owns all of its device memory (allocated in agimp_create,
 *    freed in agimp_destroy).  A handle is not thread-safe; distinct handles are
 *    independent.
 *  - Status codes are returned, never raised.  agimp_last_error() gives a
 *    message for the last failing call on a handle.
 */
#ifndef AGIMP_H
#define AGIMP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AGIMP_ABI_VERSION 2

typedef enum {
  AGIMP_OK = 0,
  AGIMP_INVALID_ARG = 1,
  AGIMP_CAPACITY = 2,
  AGIMP_NAN = 3,
  AGIMP_DEVICE_TIMEOUT = 4,
  AGIMP_CUDA_ERROR = 5,
  AGIMP_NOT_READY = 6,
  AGIMP_OUT_OF_MEMORY = 7
} agimp_status;

enum { AGIMP_MEM_DEVICE = 0, AGIMP_MEM_HOST = 1 };

/* Device error word bits (agimp_errors).  The library records these instead of
 * faulting; each names a condition the reference leaves undefined. */
#define AGIMP_ERR_OOB 1u      /* an index left the stored lattice; access skipped */
#define AGIMP_ERR_ESCAPED 2u  /* a particle left [0,1)^dim; it is frozen (fl_p = -1) */
#define AGIMP_ERR_MAP_OOB 4u  /* a level-map lookup left the table */
#define AGIMP_ERR_NOBIN 8u    /* a particle's bin block was not active (internal) */
#define AGIMP_ERR_WAIT 16u    /* a bounded device wait (tensor-core completion) gave up */

/* Mask flags, utils.py:5-9. */
#define AGIMP_ACTIVATED 1
#define AGIMP_GHOST 2
#define AGIMP_T_JUNCTION 4

/* Simulator parameters.  agimp_default_params() fills the reference's
 * constants (adaptive_gimp.py:17-18, 48-53): radius 0.5 cells, gravity
 * (0,-100,0), E 5e3, nu 0.2, boundary_gap 4 finest cells, per-axis wall clamp,
 * no plasticity, no colliders. */
typedef struct agimp_params {
  int32_t dim;            /* 2 or 3 (adaptive_gimp.py:12) */
  int32_t level;          /* number of levels L, 1..8 (adaptive_gimp.py:14) */
  int32_t coarsest_size;  /* power of two >= 4 (adaptive_gimp.py:15) */
  int32_t boundary_gap;   /* finest cells (adaptive_gimp.py:18) */
  int32_t boundary_mode;  /* 0: per-axis normal clamp (adaptive_gimp.py:284-287); 1: sticky walls */
  int32_t plasticity;     /* 0: none (reference); 1: snow (Stomakhin et al. 2013), extension */
  int64_t n_particles;    /* adaptive_gimp.py:51 */
  double radius;          /* GIMP half-width in cells (adaptive_gimp.py:48) */
  double gravity[3];      /* adaptive_gimp.py:50 */
  double E, nu;           /* adaptive_gimp.py:52-53 */
  double theta_c, theta_s, hardening; /* snow parameters (extension) */
  int32_t n_colliders;    /* sticky box colliders, extension, <= 4 */
  double colliders[4][6]; /* lo[3], hi[3] in domain units */
  /* Grid nodes that receive P2G mass but are neither activated, ghost nor
   * T-junction nodes.  0 (reference, adaptive_gimp.py:280): the grid update
   * skips them, so G2P reads their unnormalised momentum.  1 (extension):
   * their momentum is divided by their mass (no gravity, no walls), which
   * keeps dense particle regions on coarse levels stable. */
  int32_t invalid_nodes;
} agimp_params;

typedef struct agimp_stats {
  int32_t active_blocks[8]; /* 4^dim-cell blocks visited per level in the last substep */
  int32_t n_binned;         /* particles with fl_p >= 0 in the last substep */
  int32_t n_chunks;         /* P2G/G2P work items in the last substep */
  int64_t substeps;         /* substeps run since creation */
  int32_t n_surrogate;      /* particles whose return map went to the surrogate MLP (last substep) */
  int32_t n_fallback;       /* of those, predictions rejected for the exact return map */
} agimp_stats;

typedef struct agimp_sim agimp_sim;

int agimp_abi_version(void);
const char* agimp_status_string(agimp_status s);

/* Reference constants for (dim, level, coarsest_size, n_particles). */
void agimp_default_params(agimp_params* p, int32_t dim, int32_t level, int32_t coarsest_size, int64_t n_particles);

/* Replaces AdaptiveGIMP.__init__ storage and constants (adaptive_gimp.py:6-62).
 * Allocates every device buffer for the dense blocked lattices of all levels
 * and the particle arrays; nothing is allocated afterwards. */
agimp_status agimp_create(const agimp_params* p, int32_t device, agimp_sim** out);
agimp_status agimp_destroy(agimp_sim* s);
const char* agimp_last_error(const agimp_sim* s);

/* Replaces the particle_initializer hook (adaptive_gimp.py:64, init.py:3-32):
 * writes x_p, v_p, F_p, C_p, m_p, g_p (adaptive_gimp.py:55-61) and, with snow
 * plasticity, Jp (NULL = 1).  Any array may be NULL to leave it unchanged. */
agimp_status agimp_set_particles(agimp_sim* s, const float* x, const float* v, const float* F, const float* C,
                                 const float* m, const int32_t* g, const float* Jp, int32_t memory, void* stream);

/* Field readback of x_p, v_p, F_p, C_p, m_p, g_p, fl_p (adaptive_gimp.py:55-62)
 * and Jp.  NULL outputs are skipped. */
agimp_status agimp_get_particles(agimp_sim* s, float* x, float* v, float* F, float* C, float* m, int32_t* g,
                                 int32_t* fl, float* Jp, int32_t memory, void* stream);

/* The bins of the last substep (adaptive_gimp.py:208-216, the pid[l] lists:
 * particle p sits in the list of level fl_p at block base // 4 of that
 * level), one key per particle in the caller's order: the level in bits 60-63
 * and, per axis, floor(base / 4) + 1 in a 20-bit field (first axis highest);
 * UINT64_MAX for particles without a level (fl_p = -1).  Particles with equal
 * keys share a pid block.  AGIMP_NOT_READY until a substep has binned the
 * current state (after agimp_set_particles, or before the first substep). */
agimp_status agimp_get_bins(agimp_sim* s, uint64_t* keys, int32_t memory, void* stream);

/* Asynchronous field readback into HOST memory (pinned, for the copy to
 * overlap): enqueues the copy of the current state on `stream` and returns at
 * once; the outputs hold the state once `stream` has run the enqueued work
 * (synchronize it or wait on an event recorded after the call).  No counterpart
 * in the reference (Taichi's to_numpy blocks).  The copy waits for the
 * substeps, uploads and refinements already issued, and later ones that
 * would overwrite the state being copied wait for the fields to be gathered
 * into a staging slot (a short kernel on the library's own stream, behind the
 * state and the slot's previous host copy only), whatever streams they use:
 * the state of substep k can be read while substep k+1 runs, and its host
 * copy can overlap substeps k+1 and k+2.  Allocates its staging (two slots of
 * N x the requested components floats) on first use, and again when a call
 * requests more fields. */
agimp_status agimp_get_particles_async(agimp_sim* s, float* x, float* v, float* F, float* C, float* m, int32_t* g,
                                       int32_t* fl, float* Jp, void* stream);

/* Replaces the grid_initializer hook and static adaptivity
 * (adaptive_gimp.py:65-66, 72-85; init.py:34-98).  `table` tabulates the
 * initializer over finest cells [-halo, finest+halo)^dim, first axis slowest:
 * low 4 bits = the level it returns; bit 6 set = it activates nothing (else it
 * activates the cell of that level containing the finest cell).
 * halo must be >= max(2, 2^(level-1)).  Selecting a map switches the substep
 * to static activation; agimp_clear_level_map() switches back to dynamic
 * activation from g_p (adaptive_gimp.py:87-96). */
agimp_status agimp_set_level_map(agimp_sim* s, const int8_t* table, int32_t halo, int32_t memory, void* stream);
agimp_status agimp_clear_level_map(agimp_sim* s);
/* Readback of the selected level map: *halo, and when table is not null the
 * (finest + 2 halo)^dim entries in the layout agimp_set_level_map takes. */
agimp_status agimp_get_level_map(agimp_sim* s, int8_t* table, int32_t* halo, int32_t memory, void* stream);

/* Replaces AdaptiveGIMP.substep(dt0) (adaptive_gimp.py:323-352), run n_steps
 * times back to back.  Asynchronous on `stream`.  With graphs enabled (the
 * default) the substep is captured as a CUDA graph once per stream (and per
 * particle buffer, which alternates between substeps) and replayed; dt and
 * the other settings live in device memory, so changing them needs no new
 * capture. */
agimp_status agimp_substep(agimp_sim* s, float dt, int32_t n_steps, void* stream);
agimp_status agimp_set_graphs(agimp_sim* s, int32_t enable);

/* Extension with no counterpart in the reference (which fixes g_p once, in
 * init.py:17-29 / run_3d.py:151-156): recompute g_p from the current positions.
 * A particle whose finest cell is within `band` finest cells (Chebyshev) of an
 * empty finest cell gets the finest level, within band*3 the next coarser,
 * band*7 the next, ..., deeper particles level 0.  Depths are kept in bytes:
 * band * (2^(levels-1) - 1) must be below 250 (band in [1, 32]), else
 * AGIMP_INVALID_ARG. */
agimp_status agimp_refine_levels(agimp_sim* s, int32_t band, void* stream);

/* Readback of cell_mask[l], ad_grid_m[l], ad_grid_v[l] (adaptive_gimp.py:35-42)
 * as they stand after the last substep, over indices [lo, lo+n)^dim.  v is
 * [n^dim][dim].  NULL outputs are skipped. */
agimp_status agimp_get_grid(agimp_sim* s, int32_t level, int32_t lo, int32_t n, float* m, float* v, int32_t* cell_mask,
                            int32_t memory, void* stream);

/* Readback of node_mask over the finest lattice [0, finest]^dim
 * (adaptive_gimp.py:23-26); the predicates of adaptive_gimp.py:126-140 apply
 * to it unchanged. */
agimp_status agimp_get_node_mask(agimp_sim* s, int32_t* out, int32_t memory, void* stream);

/* Device error word (AGIMP_ERR_*) accumulated since the last clear.
 * Synchronizes the device. */
agimp_status agimp_errors(agimp_sim* s, uint32_t* bits, int32_t clear);
agimp_status agimp_get_stats(agimp_sim* s, agimp_stats* out);

/* Number of kernels one substep launches (for launch accounting). */
int32_t agimp_kernels_per_substep(const agimp_sim* s);

/* One substep with direct launches and CUDA events between its phases;
 * writes 8 durations in ms: active blocks, topology, binning, P2G,
 * restriction, grid_op, prolongation, G2P.  Synchronizes the stream.  The
 * reference's closest counterpart is the Taichi kernel profiler
 * (run_3d.py:12, 43). */
agimp_status agimp_profile_substep(agimp_sim* s, float dt, float* ms, int32_t n, void* stream);

/* No counterpart in the reference.  The refinement rule of
 * agimp_refine_levels for callers that cannot allocate device memory (a host
 * whose own arena or pool owns the device memory, so a library cudaMalloc
 * would fail or bypass its accounting, or a loop that cannot take the
 * synchronisation cudaMalloc/cudaFree may imply).  It takes no handle and
 * allocates nothing: x [n][dim] f32 and g [n] i32 are caller device buffers,
 * and its scratch is a static 16 MiB device array inside libagimp.so, held by
 * every GPU that loads the library until exit, which limits it to
 * finest^dim <= 16,777,216 cells (3D 256^3, 2D 4096^2); larger grids return
 * AGIMP_CAPACITY.  band and level obey agimp_refine_levels' limit
 * (band * (2^(level-1) - 1) below 250).  The first call on a device looks up the array's device
 * address with that device current; make that first call before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race.
 * Asynchronous on `stream`. */
agimp_status agimp_refine_levels_noalloc(const float* x, int64_t n, int32_t dim, int32_t level, int32_t coarsest_size,
                                         int32_t band, int32_t* g, void* stream);

/* ---- Surrogate return-map MLP (extension; the reference has no plasticity) ----
 * 7 inputs -> 64 -> 64 -> 4 outputs, SiLU after both hidden layers, bf16
 * weights and activations with f32 accumulation on the tensor cores
 * (tcgen05).  Parameters are one f32 vector of agimp_mlp_num_params() values:
 * W1[7][64], b1[64], W2[64][64], b2[64], W3[64][4], b3[4] (row-major, y = x W + b).
 * X [n][7] and Y [n][4] are device arrays. */
typedef struct agimp_mlp agimp_mlp;
int32_t agimp_mlp_num_params(void);
agimp_status agimp_mlp_create(int32_t device, agimp_mlp** out);
agimp_status agimp_mlp_destroy(agimp_mlp* m);
agimp_status agimp_mlp_set_params(agimp_mlp* m, const float* params, int32_t memory, void* stream);
agimp_status agimp_mlp_get_params(agimp_mlp* m, float* params, int32_t memory, void* stream);
agimp_status agimp_mlp_forward(agimp_mlp* m, const float* X, float* Y, int64_t n, void* stream);
/* Loss (mean over the n samples of the squared error summed over the 4
 * outputs) and its gradient with respect to the parameters, both computed on
 * the tensor cores; grad [num_params] and loss [1] are device arrays (either
 * may be NULL).  T [n][4] holds the targets. */
agimp_status agimp_mlp_grad(agimp_mlp* m, const float* X, const float* T, int64_t n, float* grad, float* loss,
                            void* stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the full batch; loss
 * (device, may be NULL) receives the loss before the step. */
agimp_status agimp_mlp_train_step(agimp_mlp* m, const float* X, const float* T, int64_t n, float lr, float* loss,
                                  void* stream);
agimp_status agimp_mlp_reset_optimizer(agimp_mlp* m);

/* Surrogate return map in the substep (snow plasticity only).  Particles whose
 * trial singular values leave the clamp interval get an SVD as before; their
 * features (see snow_features in csrc/common.cuh) go through the MLP, whose
 * prediction is used unless a feature lies outside the trained range
 * |x_k| <= xmax[k] (k < 7, host array) or the prediction's residual (distance
 * from the clamp interval, or the plastic-volume balance error in log Jp)
 * exceeds tol; those particles take the exact return map.  m must outlive its
 * use; m == NULL switches the surrogate off.  Allocates its buffers (N x 35
 * floats) on first use. */
agimp_status agimp_set_surrogate(agimp_sim* s, const agimp_mlp* m, const float* xmax, float tol);
/* Training-pair recorder (snow plasticity): every substep, particles whose new
 * slot is a multiple of `stride` append (features [7], exact projected state
 * [4]) to the device arrays X [capacity][7], T [capacity][4]; X == NULL
 * switches it off.  agimp_recorded returns the number appended (it may exceed
 * capacity; only the first capacity are stored). */
agimp_status agimp_set_recorder(agimp_sim* s, float* X, float* T, int64_t capacity, int32_t stride);
agimp_status agimp_recorded(agimp_sim* s, int64_t* count, int32_t reset);
/* bit 0: a tensor-core completion wait timed out.  Synchronizes the device. */
agimp_status agimp_mlp_errors(agimp_mlp* m, uint32_t* bits, int32_t clear);
/* No counterpart in the reference (Taichi has no device-side waits): a
 * self-test of the bounded completion wait every tensor-core kernel uses.
 * One CTA waits on an mbarrier; with arrive != 0 a thread arrives first and the
 * wait succeeds (AGIMP_OK, *bits = 0); with arrive == 0 nothing arrives, the
 * wait gives up after max_polls polls, the kernel records the timeout and
 * returns normally: AGIMP_DEVICE_TIMEOUT and *bits = AGIMP_ERR_WAIT, with the
 * CUDA context still usable.  Synchronizes the device. */
agimp_status agimp_wait_selftest(int32_t device, int32_t arrive, uint32_t max_polls, uint32_t* bits);

/* ---- Headless drawing (2D).  The reference's GUI (gui.py) draws into a GGUI
 * window; there is no window here, the image goes to a buffer.  img is
 * [res][res][3] f32 RGB indexed [i][j] like gui.py's bg_img[i, j] (i along x,
 * j along y). */
/* GUI.visualize_mask (gui.py:12-43) after the last substep: activated and
 * (show_ghost) ghost cells of every level, coarse to fine, with their edge
 * colours, then (show_node) the 3x3-pixel markers of activated, T-junction
 * and ghost finest nodes.  res >= finest size.  Where markers overlap
 * (res / finest < 3) each pixel takes the last covering node in row-major
 * order (the reference's result then depends on its thread order). */
agimp_status agimp_render_mask(agimp_sim* s, int32_t res, int32_t show_ghost, int32_t show_node, float* img,
                               int32_t memory, void* stream);
/* canvas.circles(x_p, radius, per_vertex_color=c_p) (gui.py:69) over img: a
 * pixel whose centre lies within radius * res pixels of a particle takes the
 * particle's colour (colors [N][3] in the caller's particle order; later
 * particles on top).  Allocates its scratch (res^2 ints, and an image for
 * host img) on first use. */
agimp_status agimp_render_particles(agimp_sim* s, int32_t res, float radius, const float* colors,
                                    int32_t colors_memory, float* img, int32_t memory, void* stream);

/* GUI3D.show (gui_3d.py:50-64) without a window: x_p as spheres of one
 * radius and colour (scene.particles), optionally the unit floor quad y = 0
 * (scene.mesh of bound_box), lit by point lights (scene.point_light) and an
 * ambient term, seen from a pinhole camera.  Each pixel casts a ray through
 * its centre; the nearest sphere (exact intersection; ties to the lower
 * caller index) or the floor (two-sided) is shaded with Lambert terms, no
 * shadows or specular (GGUI's own shaders are not reproduced).  The camera
 * basis is orthonormal: ray = normalise(forward + sx right + sy up) with
 * sx = (2 (col + 1/2) / res - 1) tan_half_fov, sy = (1 - 2 (row + 1/2) / res)
 * tan_half_fov.  img: [res][res][3] f32, row 0 at the top.  Spheres that reach
 * the camera's plane are not drawn.  Allocates its scratch on first use. */
typedef struct agimp_view3d {
  float eye[3], right[3], up[3], forward[3];
  float tan_half_fov; /* tan(vertical field of view / 2) */
  float radius;       /* sphere radius (scene.particles radius) */
  float color[3];     /* sphere colour */
  int32_t floor;      /* draw the floor quad [0,1] x {0} x [0,1] */
  float floor_color[3];
  float ambient[3];
  int32_t n_lights;   /* 0..4 */
  float light_pos[4][3], light_color[4][3];
  float background[3];
} agimp_view3d;
agimp_status agimp_render_scene3d(agimp_sim* s, int32_t res, const agimp_view3d* view, float* img, int32_t memory,
                                  void* stream);
/* GUI3D._draw_lines (gui_3d.py:35-47): for every cell whose mask is exactly
 * ACTIVATED, at every level, the 24 vertices [24][3] (f32) of its 12 edges in
 * the reference's stencil order (corner k = dI_0 + 2 dI_1 + 4 dI_2 at
 * (I + dI) dx).  Cells come in no fixed order.  Writes at most `capacity`
 * vertices and returns in *count the number of vertices of all cells.  3D only. */
agimp_status agimp_cell_lines(agimp_sim* s, float* vertices, int64_t capacity, int64_t* count, int32_t memory,
                              void* stream);

/* ---- Launch tuning (no counterpart in the reference: Taichi picks its own
 * launch sizes).  Results do not depend on it beyond the order of float
 * additions. */
typedef struct agimp_tuning {
  int32_t chunk;        /* particles per P2G work item (CTA size): 64, 128, 256 or 512 */
  int32_t ctas_per_sm;  /* CTAs of the grid-stride kernels per multiprocessor, 1..32 */
  float ms_per_substep; /* the autotuner's measurement of this choice (else as set) */
} agimp_tuning;
agimp_status agimp_set_tuning(agimp_sim* s, const agimp_tuning* t);
agimp_status agimp_get_tuning(const agimp_sim* s, agimp_tuning* t);
/* Measure every (chunk, ctas_per_sm) in {64, 128, 256, 512} x {2, 4, 8, 16}:
 * two warm-up and `trials` timed substeps each, all from the current state,
 * which is restored afterwards (the simulation does not advance).  Keeps and
 * returns the fastest.  Synchronizes the stream. */
agimp_status agimp_autotune(agimp_sim* s, float dt, int32_t trials, agimp_tuning* best, void* stream);

/* ---- Batches (no counterpart in the reference).  Independent simulators on
 * one device and of one dimension (any levels, sizes, particle counts, static
 * or dynamic) stepped together: every kernel of the substep is launched once
 * for all of them, and the sequence is captured as a CUDA graph.  Each
 * simulator keeps its own state and readback; stepping a batch advances all
 * of them by the same substeps, exactly as agimp_substep on each would (up to
 * the order of float additions).  The simulators must outlive the batch.  In a
 * batch of several scenes the surrogate return map is the batch's own
 * (agimp_batch_set_surrogate): the scenes' individual surrogate settings apply
 * only when they step alone. */
typedef struct agimp_batch agimp_batch;
agimp_status agimp_batch_create(agimp_sim* const* sims, int32_t n, agimp_batch** out);
agimp_status agimp_batch_destroy(agimp_batch* b);
const char* agimp_batch_last_error(const agimp_batch* b);
agimp_status agimp_batch_substep(agimp_batch* b, float dt, int32_t n_steps, void* stream);
agimp_status agimp_batch_set_graphs(agimp_batch* b, int32_t enable);
agimp_status agimp_batch_set_tuning(agimp_batch* b, const agimp_tuning* t);
agimp_status agimp_batch_get_tuning(const agimp_batch* b, agimp_tuning* t);
/* As agimp_autotune, over the whole batch. */
agimp_status agimp_batch_autotune(agimp_batch* b, float dt, int32_t trials, agimp_tuning* best, void* stream);
int32_t agimp_batch_kernels_per_substep(const agimp_batch* b);
/* Positions of all scenes in one copy: x [sum of N][dim] in HOST memory
 * (pinned, for overlap), scene after scene in batch order, each scene in its
 * caller's particle order.  Asynchronous like agimp_get_particles_async: the
 * gather into a staging slot waits for the batch's substeps already issued,
 * and the substep that overwrites that state waits for the gather (a short
 * kernel on the batch's own stream), so the host copy overlaps the next
 * substeps.  (Orders only against the batch's own steps and uploads.)
 * Allocates its staging (two slots) on first use. */
agimp_status agimp_batch_positions_async(agimp_batch* b, float* x, void* stream);
/* Upload of every scene's particles in one call (a batch of several): the
 * arrays hold all scenes' particles concatenated in batch order, each scene
 * in its caller's particle order, shaped as agimp_set_particles takes them
 * (x, v [sum of N][dim], F, C [sum of N][dim][dim], m, g, Jp [sum of N]); NULL
 * fields are skipped.  One copy and one scatter kernel per field for all
 * scenes; waits for asynchronous readbacks of the state it overwrites and
 * returns after the upload.  No counterpart in the reference. */
agimp_status agimp_batch_set_particles(agimp_batch* b, const float* x, const float* v, const float* F, const float* C,
                                       const float* m, const int32_t* g, const float* Jp, int32_t memory,
                                       void* stream);
/* As agimp_profile_substep, for one substep of the whole batch. */
agimp_status agimp_batch_profile_substep(agimp_batch* b, float dt, float* ms, int32_t n, void* stream);
/* No counterpart in the reference (which has no plasticity): the surrogate
 * return map for every snow scene of a batch of several, as
 * agimp_set_surrogate describes for one simulator.  All scenes hand their
 * projections to one set of slot buffers (allocated here, sized by the
 * scenes' total particle count), so one MLP launch and one finishing kernel
 * per substep serve the whole batch.  m == NULL switches it off. */
agimp_status agimp_batch_set_surrogate(agimp_batch* b, const agimp_mlp* m, const float* xmax, float tol);
/* Surrogate counts of the last substep over the batch: projections handed to
 * the MLP, predictions rejected (exact map used), and AGIMP_ERR_WAIT in
 * *errors if an MLP completion wait gave up.  Synchronizes the device. */
agimp_status agimp_batch_surrogate_stats(agimp_batch* b, int64_t* handed, int64_t* rejected, uint32_t* errors);

/* ---- Scene initialisers on the device.  The reference fills x_p, v_p, F_p,
 * m_p, g_p with Taichi kernels (init.py:3-32 initialize_particle,
 * run_3d.py:14-32 init_p) and tabulates its grid initializer through
 * activate_cell (init.py:34-98).  These write the simulator's state (and its
 * level map) on the GPU from a small description, so a large scene needs no
 * host arrays and no upload.  Every particle gets F = I, C = 0, Jp = 1, and
 * its index in the generation order as the caller's index (readback returns
 * particles in that order).  Random numbers: Philox4x32-10 (Salmon et al.,
 * SC 2011) keyed by the 64-bit seed, counter = the particle's (or lattice
 * point's) index: the result does not depend on the launch shape. */
#define AGIMP_SHAPE_BOX 0
#define AGIMP_SHAPE_SPHERE 1
typedef struct agimp_shape {
  int32_t kind;        /* AGIMP_SHAPE_BOX: lo <= x < hi; AGIMP_SHAPE_SPHERE: |x - centre|^2 < radius^2 */
  int32_t level;       /* g_p of its particles */
  double lo[3], hi[3]; /* box corners */
  double centre[3], radius;
  float velocity[3];
  float mass;
} agimp_shape;
/* Points of a jittered sub-lattice inside the shapes (the synthetic
 * benchmark scenes): per_axis points per finest cell and axis, at
 * (start + i + 1/2) h with h = 1 / (finest per_axis), i over the shape's
 * bounding box [floor(lo / h), ceil(hi / h)); with jitter, each moved by
 * -h/2 + h u per axis (u uniform in [0, 1), 53 bits, counter (k, shape,
 * 0 / 1) for lattice point k of the shape); kept when the moved point lies
 * inside its shape.  Shapes one after another, each in row-major lattice
 * order (first axis slowest).  Positions are computed in double and rounded
 * to float once.  Count first (to create the simulator), then fill: the
 * fill requires exactly n_particles points.  At most 64 shapes. */
agimp_status agimp_lattice_count(int32_t dim, int32_t finest, int32_t per_axis, int32_t jitter, uint64_t seed,
                                 const agimp_shape* shapes, int32_t n_shapes, int64_t* count, int32_t device);
agimp_status agimp_lattice_fill(agimp_sim* s, int32_t per_axis, int32_t jitter, uint64_t seed,
                                const agimp_shape* shapes, int32_t n_shapes, void* stream);
/* init.py:3-32 / run_3d.py:14-32: `count` particles per box, consecutive
 * boxes in order (the reference's two halves of the particle range), at
 * x = u size + lo in float (u uniform in [0, 1)^dim, 24 bits, counter
 * (index, 0, 0, 0)); g_p = band_level[k] of the first band k with
 * band_lo[k] <= u_d <= band_hi[k] on every axis, else `level` (the
 * reference's `if all(0.2 <= xy <= 0.8)` chain).  The counts must sum to
 * n_particles.  At most 16 boxes. */
typedef struct agimp_random_box {
  int64_t count;
  float lo[3], size[3];
  float velocity[3];
  float mass;
  int32_t n_bands; /* 0..4 */
  float band_lo[4], band_hi[4];
  int32_t band_level[4];
  int32_t level;
} agimp_random_box;
agimp_status agimp_random_fill(agimp_sim* s, uint64_t seed, const agimp_random_box* boxes, int32_t n_boxes,
                               void* stream);
/* initialize_mask1..5 (init.py:34-98) tabulated on the device: the same table
 * agimp_set_level_map takes, over finest cells [-halo, finest + halo)^dim with
 * halo = max(2, 2^(level-1)).  Rules 2, 4 and 5 use level 3 and need 4 levels,
 * rule 3 needs 3. */
agimp_status agimp_set_level_map_rule(agimp_sim* s, int32_t rule, void* stream);
/* A level map constant on each coarsest cell: a finest cell inside the domain
 * gets coarse_levels[its coarsest cell] (activating), the halo level-1 without
 * activation.  coarse_levels: coarsest_size^dim int8, first axis slowest. */
agimp_status agimp_set_coarse_level_map(agimp_sim* s, const int8_t* coarse_levels, int32_t memory, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AGIMP_H */
