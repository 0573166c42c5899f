/*
 * ckmpm.h -- C ABI of the B200-native CK-MPM substep engine.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes.  No
 * exit()/abort(); every failure is reported through the status and
 * ckmpm_last_error().  One host thread per scene handle; all device memory is
 * owned by the handle and released by ckmpm_destroy().
 *
 * The entry points replace the reference's header-only C++ API
 * (AppledoreM/CKMPM, include/mpm_engine.cuh), which is a per-GridConfig
 * singleton that owns its device memory, ends the process on errors and on
 * completion, and takes its scene constants from compile-time CRTP classes
 * (include/mpm_config.h:12-124).  Here the same constants travel in
 * ckmpm_scene_desc at run time.
 */
#ifndef CKMPM_H_
#define CKMPM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ckmpm_scene ckmpm_scene;

typedef enum ckmpm_status {
  CKMPM_OK = 0,
  CKMPM_ERR_INVALID = 1,   /* bad argument or call order */
  CKMPM_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  CKMPM_ERR_CAPACITY = 3,  /* a block or the block table overflowed */
  CKMPM_ERR_NUMERIC = 4,   /* non-finite or out-of-range values on the grid */
  CKMPM_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
  CKMPM_ERR_NOT_FOUND = 6  /* no such model / buffer too small */
} ckmpm_status;

/* Constitutive models; the numbering follows MPMConstitutiveModel
 * (include/mpm_material.cuh:10-18). */
typedef enum ckmpm_material_kind {
  CKMPM_FIXED_COROTATED = 0,
  CKMPM_LINEAR = 1,
  CKMPM_DRUCKER_PRAGER = 2,
  CKMPM_FLUID = 3,
  CKMPM_VON_MISES = 4,
  CKMPM_NACC = 5 /* kNonAssociatedCamClay */
} ckmpm_material_kind;

/* Grid boundary rules.  STICKY_BLOCKS is the reference's built-in rule: every
 * grid block within two blocks of the domain edge gets zero velocity
 * (include/mpm_algorithm.cuh:765-768,802-805).  SLIP_FLOOR keeps sticky x/z
 * walls and ceiling, and clamps v_y >= 0 for cells below floor_cells (the
 * per-cell hook a scene installs through ProcessGridCellVelocity,
 * include/mpm_config.h:108-117).  FIELD takes one rule per grid cell from
 * ckmpm_set_boundary_field: the reference's irregular-boundary hook
 * (GetExistIrregularBoundary / ProcessGridCellVelocity, include/mpm_algorithm.cuh:795-799)
 * evaluated into data, so scene hooks such as slip walls, fixed regions or
 * driven grips run without scene code on the device. */
typedef enum ckmpm_boundary_kind {
  CKMPM_BOUNDARY_STICKY_BLOCKS = 0,
  CKMPM_BOUNDARY_SLIP_FLOOR = 1,
  CKMPM_BOUNDARY_FIELD = 2
} ckmpm_boundary_kind;

/* Per-cell rules of CKMPM_BOUNDARY_FIELD, applied to a grid node's velocity
 * after gravity when its mass exceeds the clamp (both staggered grids of a cell
 * take the cell's rule, as the reference's hook sees only the cell index).
 * param is a unit normal n (SLIP, SEPARATE) or a velocity u (VELOCITY). */
typedef enum ckmpm_cell_rule {
  CKMPM_CELL_FREE = 0,      /* no constraint */
  CKMPM_CELL_FIXED = 1,     /* v = 0 */
  CKMPM_CELL_SLIP = 2,      /* v -= (n . v) n */
  CKMPM_CELL_VELOCITY = 3,  /* v = u */
  CKMPM_CELL_SEPARATE = 4   /* if n . v < 0: v -= (n . v) n */
} ckmpm_cell_rule;

/* Scene constants: the getters of MPMConfigBase (include/mpm_config.h:17-123)
 * and the block extent of MPMDomainRange (include/mpm_domain.h:17-30). */
typedef struct ckmpm_scene_desc {
  float dx;                  /* cell size; GetDx() */
  int32_t domain_blocks[3];  /* domain extent in 4^3-cell blocks; MPMDomainRange<Bx,By,Bz> */
  float gravity;             /* acceleration along y; GetGravity() */
  float mass_clamp;          /* nodes with m <= mass_clamp get v = 0; GetMassClamp() */
  int32_t boundary;          /* ckmpm_boundary_kind */
  float floor_cells;         /* slip-floor height in cells (SLIP_FLOOR only) */
  uint32_t max_particles_per_block; /* capacity per 4^3 block (reference: 64 per cell x 64 cells); <= 4096 */
  int32_t device;            /* CUDA device ordinal */
  uint32_t flags;            /* CKMPM_FLAG_* */
} ckmpm_scene_desc;

/* Keep a per-particle original index so state can be returned in input order. */
#define CKMPM_FLAG_TRACK_IDS 1u

/* Material parameters in the field order of each MPMMaterial<k>::MaterialParameter_
 * (include/mpm_material.cuh:24-257):
 *   FIXED_COROTATED, DRUCKER_PRAGER, LINEAR: p[0] = lambda, p[1] = mu;
 *   FLUID: p[0] = bulk, p[1] = gamma, p[2] = viscosity, p[3] = J0;
 *   VON_MISES: p[0] = mu, p[1] = lambda, p[2] = yield stress;
 *   NACC: p[0] = mu, p[1] = lambda, p[2] = alpha0 (initial logJp), p[3] = beta,
 *         p[4] = hardening factor, p[5] = M, p[6] = hardening on (0 or 1).
 * Unused entries are ignored. */
typedef struct ckmpm_material {
  int32_t kind; /* ckmpm_material_kind */
  float p[8];
} ckmpm_material;

/* Replaces MPMEngine<GridConfig>::GetInstance() + Initialize(config)
 * (include/mpm_engine.cuh:80-84,171-191).  Allocates the scene's dense grids,
 * stamps and scalars in one device allocation.  Each scene also takes one
 * page-locked host word (its export count) from slabs of 1024 that the
 * library allocates as needed (64 KB each) and keeps for the life of the
 * process; ckmpm_destroy returns the word. */
ckmpm_status ckmpm_create(const ckmpm_scene_desc* desc, ckmpm_scene** out);

/* Replaces MPMModel(mass, volume, x, v, material) (include/mpm_model.h:19-33)
 * plus the per-model part of MPMEngine::InitializeParticle
 * (include/mpm_engine.cuh:92-168).  x: n float3 positions, v: nv float3
 * velocities with nv == 1 (shared) or nv == n.  Host pointers; they are
 * copied to the device before the call returns (by DMA when pinned). */
ckmpm_status ckmpm_add_model(ckmpm_scene* s, const ckmpm_material* material, uint32_t n, const float* x,
                             const float* v, uint32_t nv, float mass, float volume, int32_t* model_index);

/* Replaces MPMEngine::InitialSetup (include/mpm_engine.cuh:216-383): first
 * binning, block table, initial state (F = I, logJp = 0, J = J0) and the
 * initial mass/momentum grid.  The next substep advects with dt = 0, as the
 * reference's first Simulate step does (include/mpm_engine.cuh:479-480). */
ckmpm_status ckmpm_setup(ckmpm_scene* s);

/* Replaces the body of MPMEngine::Simulate's substep loop
 * (include/mpm_engine.cuh:519-876) with the step size fixed: runs nsteps
 * substeps where each advects with the previous substep's dt and deposits
 * stress with `dt` (the reference's currentDt / nextDt pair).  Asynchronous on
 * the scene's stream except for one status read at the end. */
ckmpm_status ckmpm_step(ckmpm_scene* s, uint32_t nsteps, float dt);

/* Same as ckmpm_step, but enqueues only: no synchronisation and no status
 * read; call ckmpm_status_check() later. */
ckmpm_status ckmpm_step_async(ckmpm_scene* s, uint32_t nsteps, float dt);

/* Synchronise the scene's stream and turn the device status word into a code. */
ckmpm_status ckmpm_status_check(ckmpm_scene* s);

/* Adaptive step, the reference's CFL rule (include/mpm_engine.cuh:552-557):
 * next dt = min(dt_max, frame_remaining, dx * cfl / max|v_grid|), computed on
 * the device from the grid of the previous substep.  Advances nsteps substeps
 * and returns the simulated time in *elapsed (may be NULL).  frame_time = 0
 * continues the frame an earlier call opened (stepping one substep at a time). */
ckmpm_status ckmpm_step_adaptive(ckmpm_scene* s, uint32_t nsteps, float dt_max, float cfl, double frame_time,
                                 double* elapsed);

/* Rigid particles, the reference's scene hooks GetExistRigidParticle,
 * GetRigidParticleCount and GetRigidParticleVelocity(frame)
 * (include/mpm_config.h:92-106) as used by its particle initialisation
 * (include/mpm_algorithm.cuh:1063-1069) and G2P2G (:1540-1543, :1609-1624).
 * ckmpm_set_rigid, before ckmpm_setup, turns them on: the first rigid_count
 * input particles of every von Mises model start rigid (aux = 0).  As in the
 * reference, every particle whose bucket attribute 3 is exactly zero is then
 * rigid (F00 for fixed-corotated, Drucker-Prager and linear, J for the fluid,
 * logJp for NACC, the flag for von Mises): it moves by dt * velocity, deposits
 * its mass with zero momentum and zero affine field, and reports v = 0.  Not
 * for a batch.  ckmpm_set_rigid_velocity changes the velocity for the
 * substeps enqueued after it (the reference evaluates its hook per frame). */
ckmpm_status ckmpm_set_rigid(ckmpm_scene* s, uint32_t rigid_count, const float* velocity3);
ckmpm_status ckmpm_set_rigid_velocity(ckmpm_scene* s, const float* velocity3);

/* The per-cell boundary of a CKMPM_BOUNDARY_FIELD scene.  rule: one
 * ckmpm_cell_rule byte per cell of the domain (4 * domain_blocks cells per
 * axis, index (cx * Ny + cy) * Nz + cz); param: 3 floats per cell in the same
 * order, or NULL when every rule is FREE or FIXED.  Host arrays.  Before
 * ckmpm_setup, or later to change the boundary for the substeps enqueued after
 * the call (the reference's hook also receives the frame index).  The scenes
 * of a batch share one field. */
ckmpm_status ckmpm_set_boundary_field(ckmpm_scene* s, const uint8_t* rule, const float* param);

/* Use a caller-provided cudaStream_t (passed as void*) for all work of this
 * scene; NULL selects the scene's own stream. */
ckmpm_status ckmpm_set_stream(ckmpm_scene* s, void* cuda_stream);

/* Number of live particles of a model (after losses to the domain edge). */
ckmpm_status ckmpm_get_count(ckmpm_scene* s, int32_t model, uint32_t* n_live);

/* Per-particle state, replacing the export path's RetrieveParticleBuffer +
 * D2H (include/mpm_algorithm.cuh:1977-2020, include/mpm_engine.cuh:386-454).
 * Arrays hold n_live entries (x, v: 3 floats; F: 9 floats row-major, the
 * identity for the fluid; aux: J for the fluid, logJp for Drucker-Prager and
 * NACC, the rigid flag for von Mises (1 deformable, 0 rigid), 0 otherwise;
 * id: input index).  With
 * CKMPM_FLAG_TRACK_IDS the arrays are in input order and id is the identity
 * over live particles; without it they are in block order.  v is the velocity
 * the next G2P interpolates at each particle (the reference's conservation
 * probe, include/mpm_algorithm.cuh:1306-1331).  Any pointer may be NULL.
 * Host pointers; cap is the capacity in particles. */
ckmpm_status ckmpm_get_state(ckmpm_scene* s, int32_t model, float* x, float* v, float* F, float* aux,
                             uint32_t* id, uint32_t cap, uint32_t* n_out);

/* Positions export that overlaps the substeps enqueued after it, in place of
 * the reference's per-frame ExportParticleToModel + background exporter
 * thread (include/mpm_engine.cuh:386-454, include/mpm_io.h:93-166).  Enqueues
 * on the scene's stream the gather of model's positions as ckmpm_get_state
 * writes x (input order with CKMPM_FLAG_TRACK_IDS, else block order) into a
 * device staging buffer, then copies it into x on a second stream; returns
 * without waiting.  x is a host buffer (pinned, for the copy to overlap) of
 * cap >= the model's particle count floats x 3; it must not be read before
 * ckmpm_export_wait, which waits for the last export and gives its live
 * count (the valid leading entries of x).  A later export or ckmpm_get_state
 * waits for the previous copy on the device before it reuses the staging
 * buffer. */
ckmpm_status ckmpm_export_positions_async(ckmpm_scene* s, int32_t model, float* x, uint32_t cap);
ckmpm_status ckmpm_export_wait(ckmpm_scene* s, uint32_t* n_out);

/* Canonical block sets (what MPMPartition holds after a substep,
 * include/mpm_partition.cuh:37-174 and include/mpm_engine.cuh:659-865):
 * which = 0: blocks holding particles of `model` (all models if model < 0),
 * lexicographically sorted, with per-block particle counts in `counts`;
 * which = 1: plus their {0,1}^3 neighbours (Neighbor policy); which = 2: plus
 * their {-1,0,1}^3 neighbours (Exterior policy).  keys: int32 triples. */
ckmpm_status ckmpm_get_blocks(ckmpm_scene* s, int32_t model, int32_t which, int32_t* keys, uint32_t* counts,
                              uint32_t cap, uint32_t* n_out);

/* Device counters: [0] substeps taken, [1] particles lost at the domain edge,
 * [2] P2G window escapes (particle skipped in P2G, include/mpm_algorithm.cuh:1670-1683),
 * [3] status bits, [4] bounded-wait timeouts (the substep has no device-side waits; kept for the ABI, 0). */
ckmpm_status ckmpm_get_counters(ckmpm_scene* s, uint64_t* out5);

/* Current dt pair: [0] the dt the next substep advects with, [1] the dt it deposits stress with. */
ckmpm_status ckmpm_get_dt(ckmpm_scene* s, float* out2);

/* Simulated time in double, as the reference keeps its clock (currentTimestamp_,
 * include/mpm_engine.cuh:514-552): [0] the sum of the dt every substep advanced
 * with, [1] the end of the frame the last ckmpm_step_adaptive opened. */
ckmpm_status ckmpm_get_time(ckmpm_scene* s, double* out2);

/* Run nsteps substeps without graphs, timing every kernel with CUDA events on
 * the scene's stream.  ms_out[0]: total of the fused G2P2G launches, [1]: total
 * of the rebinning launches, [2]: number of fused launches. */
ckmpm_status ckmpm_step_profiled(ckmpm_scene* s, uint32_t nsteps, float dt, double* ms_out3);

/* One scene decomposed over ranks (no counterpart in the reference, which runs
 * on one GPU, src/cuda_util.cu:5-17).  Each rank creates the whole scene with
 * only the particles it owns; every rank then holds the whole dense grid and
 * deposits only its own particles.  After ckmpm_setup and after every single
 * substep (ckmpm_step_async with nsteps = 1), before the next one, the ranks
 * exchange the grid the next substep reads: ckmpm_dd_mark sets mask[b] = 1
 * (device int32, ckmpm_dd_blocks entries) for every domain block holding this
 * rank's deposits; the caller sums the masks over ranks and lists, in
 * increasing block order, the blocks with a sum of 2 or more (only those are
 * read by more than one rank); ckmpm_dd_pack copies the listed blocks (512
 * int64 sums, 4 KB each; zeros where this rank has no deposits) into buf; the
 * caller sums buf over ranks (an int64 all-reduce); ckmpm_dd_unpack writes the
 * sums back.  The sums are exact integers, so every rank's particles then
 * evolve bit for bit as in the undecomposed scene.  All on the scene's stream;
 * device pointers. */
ckmpm_status ckmpm_dd_blocks(ckmpm_scene* s, uint32_t* n_blocks);
ckmpm_status ckmpm_dd_mark(ckmpm_scene* s, int32_t* mask);
ckmpm_status ckmpm_dd_pack(ckmpm_scene* s, const int32_t* blocks, uint32_t n, long long* buf);
ckmpm_status ckmpm_dd_unpack(ckmpm_scene* s, const int32_t* blocks, uint32_t n, const long long* buf);

/* Device-math test hook: applies one constitutive update to n particles on
 * the GPU exactly as the substep does (dW = I + dt C; F <- dW F; SVD; return
 * map; stress).  F (9n), aux (n) are updated in place; tau (9n) receives the
 * Kirchhoff stress; U, S, V (9n, 3n, 9n, may be NULL) receive the SVD of the
 * trial F.  Every kind but LINEAR (whose stress is stored per particle).
 * Host pointers. */
ckmpm_status ckmpm_debug_constitutive(const ckmpm_material* material, uint32_t n, const float* C, float dt,
                                      float* F, float* aux, float* tau, float* U, float* S, float* V);

/* No counterpart in the reference.  Runs one complete simulation of a single
 * model -- setup and nsteps substeps, the same kernels in the same order as
 * ckmpm_create / ckmpm_add_model / ckmpm_setup / ckmpm_step / ckmpm_get_state
 * -- without allocating any memory, for callers that cannot call cudaMalloc:
 * plugins whose host runtime owns the device memory budget through its own
 * pool, and loops that cannot take the device-wide synchronisation of an
 * allocation.  All scratch lives in one fixed __device__ array of 53.1 MB,
 * part of this library's device code, that every GPU loading this library
 * keeps until exit; limits: n <= 65536 particles and at most 4096 blocks in
 * the domain (e.g. 16^3), else CKMPM_ERR_CAPACITY.  The first call on a device
 * looks up the array's device address (thread-safe).  The call waits for its
 * own work (it synchronises cuda_stream and reads counts back to the host), so
 * it cannot be captured into a CUDA graph: on a capturing stream it returns
 * CKMPM_ERR_INVALID without enqueuing anything.  x, v (nv = 1 or n float3) and the
 * outputs x_out, v_out (3n), F_out (9n), aux_out (n) are DEVICE pointers in
 * input order (outputs may be NULL; particles lost at the domain edge read
 * NaN).  Materials: every kind but the linear model (which keeps a stored
 * stress); boundary kinds STICKY_BLOCKS and SLIP_FLOOR.  Every call reuses the
 * same array and clears what it needs: calls that overlap on the GPU race.
 * *message (may be NULL) receives a static string. */
ckmpm_status ckmpm_simulate_noalloc(const ckmpm_scene_desc* desc, const ckmpm_material* material, uint32_t n,
                                    const float* x, const float* v, uint32_t nv, float mass, float volume,
                                    uint32_t nsteps, float dt, void* cuda_stream, float* x_out, float* v_out,
                                    float* F_out, float* aux_out, uint32_t* n_live, const char** message);

/* ---- Batched scenes.  No counterpart in the reference, which runs one scene
 * per process (its MPMEngine is a per-GridConfig singleton,
 * include/mpm_engine.cuh:80-90).  A batch holds nscenes independent scenes
 * that share dx, the domain extent, gravity and the boundary rule of `desc`;
 * each scene has one model with its own material, particle mass and volume.
 * Every substep of every scene runs in the same launches (one persistent fused
 * kernel and the rebinning, captured in CUDA graphs).  A scene's results do not
 * depend on the other scenes of the batch or on the launch shape, bit for bit;
 * against the same scene run alone through ckmpm_create (whose kernel is
 * compiled per material) they agree to the last bits of x, v and F, as the two
 * compilations may fuse a multiply-add differently.  After
 * ckmpm_add_batch, the scene calls (ckmpm_setup, ckmpm_step*, ckmpm_status_check,
 * ckmpm_get_count, ckmpm_get_state, ckmpm_get_counters, ckmpm_destroy, ...)
 * take the batch handle with model 0; ckmpm_get_state returns all live
 * particles ordered by input index (ids count over the concatenated input). */
#define CKMPM_MAX_BATCH_SCENES 65536u

typedef struct ckmpm_batch_scene {
  ckmpm_material material;
  float mass;     /* per particle */
  float volume;   /* per particle */
  uint32_t n;     /* particles of this scene in the concatenated input */
} ckmpm_batch_scene;

ckmpm_status ckmpm_create_batch(const ckmpm_scene_desc* desc, uint32_t nscenes, ckmpm_scene** out);

/* x, v: float3 per particle, scenes concatenated in order (host pointers). */
ckmpm_status ckmpm_add_batch(ckmpm_scene* s, uint32_t nscenes, const ckmpm_batch_scene* scenes, const float* x,
                             const float* v);

/* ckmpm_get_blocks restricted to one scene of a batch (scene 0 for a single scene). */
ckmpm_status ckmpm_get_blocks_in(ckmpm_scene* s, uint32_t scene, int32_t model, int32_t which, int32_t* keys,
                                 uint32_t* counts, uint32_t cap, uint32_t* n_out);

/* ---- Launch shape of the fused substep kernel.  No counterpart in the
 * reference (fixed launch shapes, include/mpm_engine.cuh:519-866).  Results do
 * not depend on it: the P2G tile and the grid hold exact integer sums, so the
 * order in which blocks deposit never changes a bit. */
typedef struct ckmpm_tuning {
  uint32_t threads;      /* CTA size: 128, 192, 256 or 1024 (one CTA per SM; for small scenes) */
  uint32_t ctas_per_sm;  /* resident persistent CTAs per SM, 1..occupancy */
  uint32_t graph_chunk;  /* substeps per captured CUDA graph, even, 2..64 */
  float probe_ms;        /* ckmpm_autotune: measured ms per substep; 0 otherwise */
} ckmpm_tuning;

ckmpm_status ckmpm_set_tuning(ckmpm_scene* s, const ckmpm_tuning* t);

/* Substeps between re-layouts of each block's particles (default 128; 0 =
 * never).  Setup orders the particles of every block so that the 32 a warp
 * handles lie in 32 different cells; the substeps keep each block's order, but
 * the layout fades as particles change cells, and a re-layout restores it
 * before the next substep (it moves the state twice, about the cost of one
 * substep).  Results do not depend on it.  No counterpart in the reference. */
ckmpm_status ckmpm_set_reorder_interval(ckmpm_scene* s, uint32_t substeps);

/* max_ctas_per_sm2 (may be NULL): occupancy limit at 128 and 256 threads (at
 * 1024 threads it is 1). */
ckmpm_status ckmpm_get_tuning(ckmpm_scene* s, ckmpm_tuning* t, uint32_t* max_ctas_per_sm2);

/* Autotuner: times probe_steps substeps (rounded up to whole graphs) of this
 * scene or batch at dt for every candidate launch shape (threads x CTAs per SM
 * x graph chunk), restoring the saved state before each candidate and at the
 * end, so the simulation is left exactly as it was; applies and returns the
 * fastest, with its chunk graph already captured.  results (cap entries, may
 * be NULL) receives every candidate with its probe_ms. */
ckmpm_status ckmpm_autotune(ckmpm_scene* s, uint32_t probe_steps, float dt, ckmpm_tuning* results, uint32_t cap,
                            uint32_t* n_results, ckmpm_tuning* best);

/* ---- Checkpoints: the whole device state of a set-up scene (particles, block
 * lists, grids, counters and dt pair) copied to or from a caller-owned DEVICE
 * buffer of ckmpm_checkpoint_bytes bytes, stream-ordered on the scene's
 * stream.  No counterpart in the reference. */
ckmpm_status ckmpm_checkpoint_bytes(ckmpm_scene* s, uint64_t* bytes);
ckmpm_status ckmpm_checkpoint_save(ckmpm_scene* s, void* device_dst);
ckmpm_status ckmpm_checkpoint_restore(ckmpm_scene* s, const void* device_src);

/* ---- Differentiable rollout.  No counterpart in the reference.  A
 * fixed-corotated model of n particles (mass, volume, Poisson ratio nu; a
 * per-particle Young's modulus given as log E) advanced nsteps substeps of dt
 * on the dense grid of desc's domain (5..64 blocks per axis; the first substep
 * advects with dt = 0, as ckmpm_step after setup).  ckmpm_diff_forward keeps a
 * checkpoint every checkpoint_every substeps; ckmpm_diff_backward recomputes
 * one segment at a time from its checkpoint and runs the hand-written adjoint
 * of P2G, the grid update, G2P and the SVD-based stress.  All array arguments
 * are DEVICE pointers, float32, particle-major: x0, v0, xT, gxT, gx0, gv0 are
 * n x 3; FT, gFT are n x 3 x 3 row-major; logE, glogE are n.  Work is ordered
 * after, and results are visible to, cuda_stream (NULL: the legacy stream).
 * backward gives the gradients of <gxT, xT> + <gFT, FT> for the last forward. */
typedef struct ckmpm_diff ckmpm_diff;

ckmpm_status ckmpm_diff_create(const ckmpm_scene_desc* desc, uint32_t n, float mass, float volume, float nu,
                               uint32_t nsteps, float dt, uint32_t checkpoint_every, ckmpm_diff** out);
ckmpm_status ckmpm_diff_forward(ckmpm_diff* d, const float* x0, const float* v0, const float* logE, float* xT,
                                float* FT, void* cuda_stream);
ckmpm_status ckmpm_diff_backward(ckmpm_diff* d, const float* gxT, const float* gFT, float* gx0, float* gv0,
                                 float* glogE, void* cuda_stream);
/* Device time (ms) of the last forward [0] and backward [1]; generation counts forwards. */
ckmpm_status ckmpm_diff_timing(ckmpm_diff* d, float* ms_out2, uint64_t* generation);
const char* ckmpm_diff_last_error(const ckmpm_diff* d);
ckmpm_status ckmpm_diff_destroy(ckmpm_diff* d);

/* Replaces the process exit at the end of Simulate (include/mpm_engine.cuh:908). */
ckmpm_status ckmpm_destroy(ckmpm_scene* s);

/* Message of the last failure on this scene (or of the last failed create). */
const char* ckmpm_last_error(const ckmpm_scene* s);

/* Library version string. */
const char* ckmpm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CKMPM_H_ */
