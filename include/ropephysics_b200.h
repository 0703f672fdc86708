/*
 * ropephysics_b200.h -- C ABI of the B200-native batched XPBD Cosserat-rod step.
 *
 * This is the drop-in boundary for RopePhysics' batched GPU rod step. Every
 * entry point below replaces one reference interface, cited as file:line in
 * the reference project:
 *   crs::gpu::Batch and its free functions   src/gpu/gpu_solver.h:44-150
 *   the rod descriptors and builders         src/core/rod.h:26-170
 *   the collision world / primitives         src/core/collision.h:83-106,
 *                                            src/core/geometry.h:17-65
 *   constraint colouring                     src/core/coloring.h:22-51
 *
 * Conventions
 *   - Plain C: POD structs, pointers and sizes; no C++ or CUDA types.
 *   - Host data is double precision, exactly as the reference's Rod; the device
 *     runs FP32 (with optional FP64 decision points, see rp_precision).
 *   - Vectors are packed xyz, quaternions packed wxyz (body -> world).
 *   - Every function returns rp_status; RP_OK is 0. On failure,
 *     rp_last_error() returns a message for the calling thread.
 *   - A handle is not thread-safe; use one host thread per rp_batch.
 *   - rp_batch_step() is asynchronous on the batch's stream (the reference's
 *     Batch::step is asynchronous on the default stream); download/read calls
 *     synchronize that stream first.
 */
#ifndef ROPEPHYSICS_B200_H
#define ROPEPHYSICS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RP_ABI_VERSION 1

typedef enum rp_status {
    RP_OK = 0,
    RP_ERR_INVALID = 1,       /* malformed argument or descriptor */
    RP_ERR_NO_DEVICE = 2,     /* no usable CUDA device (reference: create() false) */
    RP_ERR_SHARED_MEMORY = 3, /* a rod does not fit the strategy's shared memory
                                 (reference: gpu_batch.cpp:173-182) */
    RP_ERR_OUT_OF_MEMORY = 4, /* device allocation failed (gpu_batch.cpp:275-311) */
    RP_ERR_CUDA = 5,          /* a CUDA call or kernel launch failed */
    RP_ERR_BUDGET = 6,        /* serving: request exceeds the HBM budget */
    RP_ERR_NOT_READY = 7      /* serving: result not available yet */
} rp_status;

/* Execution strategy (reference: crs::gpu::Strategy, gpu_solver.h:50).
 *   RP_STRATEGY_MULTI_KERNEL  accepted for source compatibility: one CTA per
 *                             rod with all state in global memory, so any rod
 *                             length runs. Results equal RP_STRATEGY_FUSED bit
 *                             for bit (same kernel code, same order).
 *   RP_STRATEGY_FUSED         the plain one-rod-per-CTA step: state resident
 *                             in shared memory for the whole step (up to the
 *                             227 KB opt-in on B200).
 *   RP_STRATEGY_BATCHED       the persistent form: rods sorted by length into
 *                             groups, several rods per CTA, warp-synchronous
 *                             colour sweeps, work queue over all SMs. */
typedef enum rp_strategy {
    RP_STRATEGY_MULTI_KERNEL = 0,
    RP_STRATEGY_FUSED = 1,
    RP_STRATEGY_BATCHED = 2
} rp_strategy;

/* Precision flags (bitwise OR). 0 = reference order: every FP32 operation in
 * the order of the reference kernel, for parity with its GPU path.
 *   RP_PRECISION_COMPENSATED  Kahan-compensated positions and frames (frames
 *                             renormalised in FP64 once per substep; uploads
 *                             keep the double inputs' rounding residuals).
 *   RP_PRECISION_FP64_CONE    the Coulomb stick/slip cap test in FP64.
 *   RP_PRECISION_FP64_VERDICT near-boundary hold/slide classification in FP64.
 *   RP_PRECISION_COLORED_SELF the self-contact pool projected colour by colour
 *                             (greedy colours over shared particles) instead
 *                             of in the reference's serial pool order: the
 *                             reference's proposed speed-up for its serial
 *                             self-contact loop (REMAINING.md:14-17). A
 *                             different Gauss-Seidel order, so results differ
 *                             from every other mode; batched strategy only
 *                             (the fused and multi-kernel strategies keep the
 *                             serial order); a pool needing more than 32
 *                             colours keeps the exact level order. */
typedef enum rp_precision {
    RP_PRECISION_REFERENCE = 0,
    RP_PRECISION_COMPENSATED = 1,
    RP_PRECISION_FP64_CONE = 2,
    RP_PRECISION_FP64_VERDICT = 4,
    RP_PRECISION_COLORED_SELF = 8
} rp_precision;

/* Primitive types (reference: TPrimitive::Type, geometry.h:19). */
enum { RP_PRIM_PLANE = 0, RP_PRIM_SPHERE = 1, RP_PRIM_CAPSULE = 2, RP_PRIM_BOX = 3 };

/* Contact slot states written by rp_batch_read_contact_states. */
enum {
    RP_CONTACT_NONE = 0,      /* no contact generated for this (particle, primitive) */
    RP_CONTACT_SEPARATED = 1, /* generated (within the margin) but not pushing */
    RP_CONTACT_STICK = 2,     /* pushing; friction undid all tangential motion */
    RP_CONTACT_SLIP = 3       /* pushing; friction capped by the Coulomb cone */
};

/* Isotropic circular section (reference: RodMaterial, rod.h:26-45). */
typedef struct rp_material {
    double youngs;  /* E [Pa] */
    double poisson; /* nu */
    double density; /* rho [kg/m^3] */
    double radius;  /* r [m] */
} rp_material;

/* One rod as structure-of-arrays, double precision (reference: Rod,
 * rod.h:49-121). Counts: P particles, S frames (segments plus ghost frames),
 * St stretch constraints, B bend constraints. Arrays that may be NULL on
 * input are marked; a NULL load array means zero. */
typedef struct rp_rod_desc {
    int32_t num_particles, num_frames, num_stretch, num_bend;
    rp_material material;
    /* particles */
    double* x;              /* 3P */
    double* v;              /* 3P */
    double* inv_mass;       /* P, 0 = pinned */
    double* mass;           /* P (may be NULL) */
    double* ext_force;      /* 3P (may be NULL) */
    double* kin_velocity;   /* 3P: velocity a pinned particle moves at (may be NULL) */
    /* frames */
    double* q;              /* 4S */
    double* omega;          /* 3S, body frame */
    double* inertia;        /* 3S, body-frame diagonal */
    double* inv_inertia;    /* 3S, 0 = fixed (ghost) frame */
    double* ext_torque;     /* 3S, world frame (may be NULL) */
    /* stretch/shear constraints */
    int32_t* s_p0;          /* St */
    int32_t* s_p1;          /* St */
    int32_t* s_seg;         /* St */
    double* s_rest;         /* St */
    double* s_compliance;   /* 3St */
    /* bend/twist constraints */
    int32_t* b_a;           /* B */
    int32_t* b_b;           /* B */
    double* b_rest;         /* B */
    double* b_compliance;   /* 3B */
    double* b_rest_darboux; /* 3B */
} rp_rod_desc;

/* Analytic primitive (reference: TPrimitive, geometry.h:17-65). */
typedef struct rp_primitive {
    int32_t type;
    int32_t reserved;
    double a[3];            /* plane point / sphere centre / capsule end A / box centre */
    double b[3];            /* capsule end B */
    double normal[3];       /* plane unit normal */
    double half_extents[3]; /* box */
    double rotation[4];     /* box orientation, wxyz */
    double radius;          /* sphere / capsule */
    double friction;
} rp_primitive;

/* Collision world (reference: CollisionWorld, collision.h:83-106). At most 64
 * primitives per world (the batched kernel culls them per rod with a 64-bit
 * mask); the reference has no limit. */
typedef struct rp_world {
    const rp_primitive* primitives;
    int32_t num_primitives;
    int32_t self_collision;
    double self_friction;
    int32_t self_skip;            /* default 2 */
    int32_t hash_table_size;      /* default 4096 (use a small table, e.g. 256) */
    double contact_margin_radii;  /* default 0.25 */
} rp_world;

/* Step parameters (reference: BatchParams, gpu_solver.h:52-60). */
typedef struct rp_step_params {
    float dt;
    int32_t substeps;
    int32_t iterations;
    float gravity[3];
    float linear_damping;
    float angular_damping;
    int32_t contact_interval;
} rp_step_params;

/* On-device drive of one rod's pinned particle (no host upload per step):
 * the particle moves along `axis` with displacement A sin(2 pi f t + phase),
 * i.e. its kinematic velocity is A 2 pi f cos(2 pi f t + phase) evaluated at
 * the start of each substep. particle < 0 disables the drive for the rod. */
typedef struct rp_drive {
    int32_t particle;
    int32_t reserved;
    float axis[3];
    float amplitude; /* [m] */
    float frequency; /* [Hz] */
    float phase;     /* [rad] */
} rp_drive;

/* On-device waypoint schedule of one rod's pinned particle: a robot gripper
 * following a motion (reference: HarnessTask::gripperAt and gripperVelocity,
 * src/apps/harness_routing.h:56-83, harness_routing.cpp:81-106). From
 * `start`, the particle passes through waypoints[0 .. count-1], taking
 * legs[k] seconds to reach waypoint k with a smoothstep u^2 (3 - 2u) within
 * the leg, then holds at the last one; its height stays `height`. A
 * controller holds each velocity for steps_per_control steps: during step s
 * (counted from when the drives are set) the kinematic velocity is
 * (P((tick + 1) T) - P(tick T)) x (1 / T) with tick = s / steps_per_control
 * and T = dt x steps_per_control, computed on the device in double with the
 * same operations and roundings as the reference's host code and stored as
 * floats -- the velocities the reference uploads once per control tick
 * (application_cases.cpp:236-248), with no upload. particle < 0 disables the
 * schedule for the rod. */
#define RP_MAX_WAYPOINTS 8
typedef struct rp_waypoint_drive {
    int32_t particle;
    int32_t count;             /* 1 .. RP_MAX_WAYPOINTS */
    int32_t steps_per_control; /* >= 1 */
    int32_t reserved;
    double dt;                 /* the step the schedule is sampled with [s] */
    double start[2];           /* x, y [m] */
    double height;             /* z [m] */
    double legs[RP_MAX_WAYPOINTS];         /* [s], > 0 */
    double waypoints[RP_MAX_WAYPOINTS][2]; /* x, y [m] */
} rp_waypoint_drive;

/* A routing board (reference: HarnessTask, harness_routing.h:29-41): the
 * cable must pass below peg A, above peg B, laid against each (within
 * peg_radius + cable_radius + lay_slack of its centre line), and through the
 * clip between its posts, down on the board (below clip_height). */
typedef struct rp_harness_board {
    double peg_a[2];
    double peg_b[2];
    double clip[2];
    double peg_radius;
    double clip_half_gap;
    double clip_height;
    double cable_radius;
    double lay_slack;
} rp_harness_board;

/* reference: HarnessTask::Outcome, harness_routing.h:85-94 */
typedef struct rp_harness_outcome {
    double score;     /* 3 on success; smooth for learning */
    double side_a;    /* signed offset of the crossing nearest peg A [m] */
    double side_b;
    double clip_miss; /* distance from the clip centre line [m] */
    uint8_t below_a;
    uint8_t above_b;
    uint8_t through_clip;
    uint8_t success;
    uint8_t reserved[4];
} rp_harness_outcome;

typedef struct rp_rod rp_rod;     /* host-side rod descriptor owned by the library */
typedef struct rp_batch rp_batch; /* device-resident batch */

/* ------------------------------------------------------------------ device */
/* reference: cudaAvailable(), deviceName(), diagnostic(), gpu_solver.h:44-48 */
int32_t rp_cuda_available(void);
rp_status rp_device_name(char* out, size_t capacity);
rp_status rp_diagnostic(char* out, size_t capacity);
/* reference: maxFusedSegments(), gpu_solver.h:150 (here with the 227 KB
 * opt-in shared memory of sm_100, for a free rod without contacts). */
int32_t rp_max_fused_segments(void);
/* No reference counterpart. The current device's FP32 throughput, measured:
 * a grid filling every SM runs `trips` x 128 independent fused multiply-adds
 * per thread (two operations each), timed with CUDA events after one
 * warm-up launch. Writes TFLOP/s to *tflops and the timed launch's
 * milliseconds to *ms (may be NULL). The batched step is bound by FP32
 * arithmetic, so this is its roofline denominator. */
rp_status rp_measure_fp32_peak(int32_t trips, double* tflops, double* ms);
/* Message of the last failure on the calling thread ("" if none). */
const char* rp_last_error(void);
int32_t rp_abi_version(void);

/* ------------------------------------------------------------------ rods */
/* reference: makeStraightRod, rod.h:126-127 */
rp_status rp_rod_create_straight(int32_t num_segments, double length, const rp_material* material,
                                 const double origin[3], const double direction[3], rp_rod** out);
/* reference: makeRodFromCenterline, rod.h:133-134 */
rp_status rp_rod_create_centerline(const double* points, int32_t num_points,
                                   const rp_material* material, const double frame_seed[3],
                                   double twist_per_length, rp_rod** out);
/* Deep copy of caller-owned arrays (any topology). */
rp_status rp_rod_create_from_desc(const rp_rod_desc* desc, rp_rod** out);
void rp_rod_destroy(rp_rod* rod);
/* Mutable view of the rod's arrays (valid until the next call that changes
 * its sizes: rp_rod_clamp_end). reference: the public fields of Rod. */
rp_status rp_rod_view(rp_rod* rod, rp_rod_desc* out);
/* reference: clampEndExact, rod.h:160; returns the ghost frame index. */
rp_status rp_rod_clamp_end(rp_rod* rod, int32_t tip, int32_t* ghost_frame);
/* reference: Rod::pinParticle, rod.h:109 */
rp_status rp_rod_pin_particle(rp_rod* rod, int32_t particle);
/* reference: setRestFromCurrent, rod.h:167 */
rp_status rp_rod_set_rest_from_current(rp_rod* rod);

/* ------------------------------------------------------------------ colouring */
/* reference: colorStretchConstraints / colorBendConstraints, coloring.h:41-42.
 * order: num_stretch (or num_bend) entries; color_start: capacity count + 1. */
rp_status rp_rod_coloring(const rp_rod_desc* rod, int32_t bend, int32_t* order,
                          int32_t* color_start, int32_t* num_colors);
/* reference: colorConstraints, coloring.h:37. resources of constraint k are
 * resources[resource_start[k] .. resource_start[k+1]). */
rp_status rp_color_constraints(int32_t count, const int32_t* resource_start,
                               const int32_t* resources, int32_t* order, int32_t* color_start,
                               int32_t* num_colors);
/* reference: selfCollisionIndexGap, collision.h:117 */
rp_status rp_self_collision_index_gap(const rp_rod_desc* rod, const rp_world* world, int32_t* gap);

/* ------------------------------------------------------------------ batch */
/* reference: Batch::create(prototype, numRods, strategy, world),
 * gpu_solver.h:81-82, gpu_batch.cpp:150-316. Every rod is a copy of the
 * prototype and collides with `world` (NULL = no contacts). */
rp_status rp_batch_create(const rp_rod_desc* prototype, int32_t num_rods, rp_strategy strategy,
                          const rp_world* world, rp_batch** out);
/* Heterogeneous batch (no reference counterpart: the reference batch shares
 * one prototype and one world). rods[i] is rod i's descriptor; rods that pass
 * the same pointer share their topology and rest data on the device.
 * world_of_rod[i] indexes `worlds` (NULL: every rod uses worlds[0], or no
 * world when num_worlds is 0). */
rp_status rp_batch_create_mixed(const rp_rod_desc* const* rods, int32_t num_rods,
                                const rp_world* worlds, int32_t num_worlds,
                                const int32_t* world_of_rod, rp_strategy strategy,
                                rp_batch** out);
/* reference: Batch::destroy / ~Batch, gpu_solver.h:83, gpu_batch.cpp:132-138 */
void rp_batch_destroy(rp_batch* batch);
/* reference: Batch::step, gpu_solver.h:85, gpu_batch.cpp:457-473 */
rp_status rp_batch_step(rp_batch* batch, const rp_step_params* params);
/* `steps` steps; when graphs are enabled (rp_batch_set_graph) the sequence is
 * replayed from a captured CUDA graph. The batched strategy runs up to its
 * tuned steps-per-launch whole steps in one launch (same results). */
rp_status rp_batch_step_many(rp_batch* batch, const rp_step_params* params, int32_t steps);
/* No reference counterpart. One step of an RP_STRATEGY_BATCHED batch, the
 * same kernel and the same results as rp_batch_step, but the step's scratch
 * (work-queue counters, start-of-substep frames under compensated
 * precision, world-contact slots, self-contact pool, hash, sort and
 * projection levels, constraint multipliers) is carved from a fixed static
 * device array of
 * RP_STATIC_SCRATCH_BYTES instead of the batch's own buffers, and the call
 * allocates no device memory. Needs 256 bytes, plus 16 x frames under
 * RP_PRECISION_COMPENSATED, plus 32 x contact slots when the batch's plan
 * keeps the slots in global memory (rods with many or large contact
 * primitives), plus, when any rod collides with itself, 64 x self-contact
 * pool entries, 4 x (2 (hash_table_size + 1) + 3 (pool capacity + 1)) per
 * such rod and 8 x stretch constraints, plus 16 x (stretch + bend
 * constraints) when params->iterations > 1, each section rounded up to 256
 * bytes; a larger batch is rejected with RP_ERR_INVALID. The batch's device must be
 * current. The first call on a device looks up the array's address, once;
 * make that first call before any stream capture. The queue counters are
 * cleared on the batch's stream before each launch; nothing else needs to
 * start at zero. The array is shared by every call on the device: calls that
 * overlap in time (other streams, threads or batches) race on it. */
#define RP_STATIC_SCRATCH_BYTES (32u << 20)
rp_status rp_batch_step_static_scratch(rp_batch* batch, const rp_step_params* params);
/* reference: Batch::synchronize, gpu_solver.h:86 */
rp_status rp_batch_synchronize(rp_batch* batch);
/* Run the batch on a caller-owned cudaStream_t (NULL = the library's own). */
rp_status rp_batch_set_stream(rp_batch* batch, void* cuda_stream);
rp_status rp_batch_set_precision(rp_batch* batch, int32_t flags);
/* Capture rp_batch_step_many sequences into CUDA graphs (1) or launch
 * directly (0, default). */
rp_status rp_batch_set_graph(rp_batch* batch, int32_t enabled);
/* Launch shape of RP_STRATEGY_BATCHED: CTA size (128 or 256 threads; rods per
 * CTA = CTA size / team size), pairs per thread (a rod of n segments gets a
 * team of about n / (2 x pairs) threads, whole warps, 32..256) and whole steps
 * per launch in rp_batch_step_many. None of them changes results.
 * cta_threads 0 selects one rod per CTA with every array staged in shared
 * memory (the RP_STRATEGY_FUSED kernel, same results), which wins for a few
 * short rods; it needs each rod's full layout to fit one CTA.
 * rp_batch_autotune times the candidate shapes on this batch with its current
 * state (restored afterwards) and keeps the fastest; steps per launch is
 * tried up to max_steps_per_launch (at most 8), then one rod per CTA. */
rp_status rp_batch_autotune(rp_batch* batch, const rp_step_params* params, int32_t max_steps_per_launch);
rp_status rp_batch_get_tuning(const rp_batch* batch, int32_t* cta_threads, int32_t* pairs_per_thread,
                              int32_t* steps_per_launch);
rp_status rp_batch_set_tuning(rp_batch* batch, int32_t cta_threads, int32_t pairs_per_thread,
                              int32_t steps_per_launch);

/* reference: Batch::download(rodIndex, Rod&), gpu_solver.h:90. Writes x, v,
 * q and omega of rod `rod` into `out`'s arrays (same topology). */
rp_status rp_batch_download(rp_batch* batch, int32_t rod, rp_rod_desc* out);
/* reference: Batch::downloadPositions, gpu_solver.h:94. Rod-major xyz floats:
 * out[(particle_offset(rod) + i) * 3 + c]; for a homogeneous batch that is
 * out[(rod * particles + i) * 3 + c], as in the reference. */
rp_status rp_batch_download_positions(rp_batch* batch, float* out, int64_t capacity_floats);
/* Rod-major quaternion frames, wxyz floats, same ordering as positions. */
rp_status rp_batch_download_frames(rp_batch* batch, float* out, int64_t capacity_floats);
/* reference: Batch::upload(const Rod&), gpu_solver.h:97 (every rod) */
rp_status rp_batch_upload(rp_batch* batch, const rp_rod_desc* rod);
/* reference: Batch::setLoads, gpu_solver.h:102 */
rp_status rp_batch_set_loads(rp_batch* batch, int32_t rod, const rp_rod_desc* source);
/* reference: Batch::uploadRod, gpu_solver.h:105 */
rp_status rp_batch_upload_rod(rp_batch* batch, int32_t rod, const rp_rod_desc* source);
/* reference: Batch::setKinematicVelocities, gpu_solver.h:109 (rod-major xyz) */
rp_status rp_batch_set_kinematic_velocities(rp_batch* batch, const float* rod_major_xyz,
                                            int64_t count_vec3);
/* reference: Batch::setMaterialScales, gpu_solver.h:114-115. Either pointer
 * may be NULL to leave that scale at its current value; n must be numRods. */
rp_status rp_batch_set_material_scales(rp_batch* batch, const float* youngs_scale,
                                       const float* friction_scale, int32_t n);
/* On-device drives, one per rod (n = numRods); NULL clears them. */
rp_status rp_batch_set_drives(rp_batch* batch, const rp_drive* drives, int32_t n);
/* Simulated time the drives are evaluated at (advanced by every step). */
rp_status rp_batch_set_time(rp_batch* batch, double time);
/* One waypoint schedule per rod (n = num_rods), replacing the sinusoidal
 * drives of rp_batch_set_drives; the schedules' step count restarts at 0.
 * NULL removes them. */
rp_status rp_batch_set_waypoint_drives(rp_batch* batch, const rp_waypoint_drive* drives, int32_t n);
/* Routing outcome of every rod's current centre line on `board`, computed on
 * the device in double exactly as the reference evaluates downloaded float
 * positions (HarnessTask::evaluate, harness_routing.cpp:108-154; called by
 * attemptsOnGpu, application_cases.cpp:251-261, after a full
 * downloadPositions). Only the n outcomes cross to the host. Synchronous. */
rp_status rp_batch_evaluate_harness(rp_batch* batch, const rp_harness_board* board,
                                    rp_harness_outcome* out, int32_t n);

/* Raw asynchronous copies between the device state and caller memory, on
 * the batch's stream (no reference counterpart: the reference copies
 * synchronously and reorders on the host). Use pinned host memory for full
 * speed and rp_batch_synchronize() before reading what was copied. Rows are
 * 16-byte float4 in particle_offset / frame_offset order:
 *   RP_STATE_POSITIONS  read   xyz_ per particle (compensated mode: the
 *                              rounded sum, without its compensation term)
 *   RP_STATE_FRAMES     read   wxyz per frame
 *   RP_STATE_CONTACTS   read   one RP_CONTACT_* byte per slot
 *   RP_STATE_KINEMATIC  write  xyz_ kinematic velocity per particle
 * `bytes` must equal the whole array's size. */
enum { RP_STATE_POSITIONS = 0, RP_STATE_FRAMES = 1, RP_STATE_CONTACTS = 2, RP_STATE_KINEMATIC = 3 };
rp_status rp_batch_read_state_async(rp_batch* batch, int32_t what, void* dst, int64_t bytes);
rp_status rp_batch_write_state_async(rp_batch* batch, int32_t what, const void* src, int64_t bytes);

/* Overlapped copies (no reference counterpart): the same arrays as
 * rp_batch_read_state_async / rp_batch_write_state_async, but the bytes cross
 * the host link on the caller's copy stream (rp_batch_set_copy_stream, a
 * cudaStream_t) while later steps run on the batch's stream. A read first
 * copies the rows on the device into a staging buffer the batch owns (after
 * the work queued so far on the batch's stream, a few tens of microseconds),
 * then to `dst` on the copy stream; a write crosses on an input stream the
 * batch owns (on the copy stream it would queue behind the previous step's
 * reads, which wait for that step) into a staging buffer and is moved into
 * place on the batch's stream before the next step. A read's host buffer
 * must stay valid until the copy stream has passed the copy (record and wait
 * an event on it), a write's until the batch's stream has passed the next
 * step; reading the same array again, or writing again, waits on the device
 * for the previous copy out of (into) the staging buffer. The first call per
 * array allocates its staging buffer. */
rp_status rp_batch_set_copy_stream(rp_batch* batch, void* cuda_stream);
rp_status rp_batch_read_state_overlapped(rp_batch* batch, int32_t what, void* dst, int64_t bytes);
rp_status rp_batch_write_state_overlapped(rp_batch* batch, int32_t what, const void* src, int64_t bytes);

/* Per (rod, particle, primitive) contact state at the end of the last step,
 * RP_CONTACT_*; layout rod-major: (particle_offset(rod) + i) * prims + k where
 * prims is the rod's primitive count. Returns the total slot count in *count. */
rp_status rp_batch_read_contact_states(rp_batch* batch, uint8_t* out, int64_t capacity,
                                       int64_t* count);
/* Self-contact pairs (segment j, segment k) of the last contact regeneration
 * of `rod`, in projection order. */
rp_status rp_batch_read_self_contacts(rp_batch* batch, int32_t rod, int32_t* pairs_jk,
                                      int32_t capacity, int32_t* count);

/* Hold/slide observation (reference: HangOutcome, apps/cable_hanging.h:68-77):
 * every `interval` steps each rod's `particle` z is compared with its z at
 * arming time; held = max rise <= tolerance. particle < 0 disarms. */
rp_status rp_batch_arm_hold_observer(rp_batch* batch, const int32_t* particle_of_rod,
                                     int32_t n, int32_t interval, double tolerance);
/* The same, with each rod's start height given by the caller (start_z, one
 * per rod; NULL = read from the device as above). The reference's outcome
 * starts from the host rod's double height (HangOutcome(rod.state.x.front().z),
 * application_cases.cpp:47-50), not from its float copy on the device. */
rp_status rp_batch_arm_hold_observer_at(rp_batch* batch, const int32_t* particle_of_rod,
                                        const double* start_z, int32_t n, int32_t interval,
                                        double tolerance);
/* max_rise (may be NULL) and held (may be NULL), one per rod; near_boundary
 * (may be NULL) flags rods whose max rise lies within float resolution of the
 * tolerance, classified in FP64 when RP_PRECISION_FP64_VERDICT is set. */
rp_status rp_batch_read_hold_verdicts(rp_batch* batch, double* max_rise, uint8_t* held,
                                      uint8_t* near_boundary, int32_t n);

/* accessors (reference: gpu_solver.h:117-130) */
int32_t rp_batch_num_rods(const rp_batch* batch);
int32_t rp_batch_num_segments(const rp_batch* batch, int32_t rod);
int32_t rp_batch_num_particles(const rp_batch* batch, int32_t rod);
int64_t rp_batch_particle_offset(const rp_batch* batch, int32_t rod);
int32_t rp_batch_num_frames(const rp_batch* batch, int32_t rod);
int64_t rp_batch_frame_offset(const rp_batch* batch, int32_t rod);
int32_t rp_batch_strategy(const rp_batch* batch);
int32_t rp_batch_stretch_colors(const rp_batch* batch);
int32_t rp_batch_bend_colors(const rp_batch* batch);
size_t rp_batch_shared_bytes_per_block(const rp_batch* batch);
int32_t rp_batch_launches_per_step(const rp_batch* batch, const rp_step_params* params);
int64_t rp_batch_self_contact_overflow(rp_batch* batch);
/* Kernel launches issued by this batch since creation (for accounting). */
int64_t rp_batch_kernel_launches(const rp_batch* batch);
/* Rods whose kernels reported an internal inconsistency (a self-contact
 * entry indexing outside its rod, which is then dropped instead of used);
 * 0 in a correct run. -1 on a failed read. */
int64_t rp_batch_error_count(rp_batch* batch);

/* ------------------------------------------------------------------ serving */
/* Continuous batching (no reference counterpart: the reference runs one
 * Batch per caller). A server owns device arenas sized by an HBM budget and a
 * worker thread. Requests -- sets of rods with a horizon in steps -- are
 * admitted first-in first-out whenever their resident state fits the budget,
 * join the rods already on the device, and advance together: every server
 * step is ONE batched launch over all resident rods of all running requests.
 * A request whose horizon is reached is read back and retired between steps,
 * freeing its memory for the next admissions. Each rod's arithmetic is that
 * of a batch holding it alone, so a request's result does not depend on what
 * it shared the device with. All functions are thread-safe. */
typedef struct rp_server rp_server;

typedef struct rp_server_config {
    uint64_t hbm_budget_bytes; /* resident-state budget for admission */
    rp_step_params params;     /* shared by every request */
    int32_t precision;         /* rp_precision flags */
    int32_t max_steps_in_flight; /* launches queued ahead of completion checks (>= 1) */
} rp_server_config;

typedef struct rp_request {
    const rp_rod_desc* const* rods;
    int32_t num_rods;
    int32_t steps;               /* horizon */
    const rp_world* worlds;      /* may be NULL with num_worlds 0 */
    int32_t num_worlds;
    int32_t reserved;
    const int32_t* world_of_rod; /* NULL: worlds[0] for every rod */
    const rp_drive* drives;      /* one per rod, or NULL */
    const float* youngs_scale;   /* one per rod, or NULL */
    const float* friction_scale; /* one per rod, or NULL */
} rp_request;

enum { RP_REQUEST_QUEUED = 0, RP_REQUEST_RUNNING = 1, RP_REQUEST_DONE = 2 };

typedef struct rp_request_info {
    int32_t state;             /* RP_REQUEST_* */
    int32_t num_rods;
    int64_t num_particles;
    int64_t resident_bytes;
    int64_t segment_substeps;  /* work of the whole horizon */
    double submit_s, admit_s, done_s; /* server clock, seconds */
} rp_request_info;

typedef struct rp_server_stats {
    int64_t submitted, admitted, completed, queued, running;
    int64_t steps_launched;
    int64_t segment_substeps;  /* completed so far */
    int64_t resident_bytes, peak_resident_bytes, budget_bytes;
    double now_s;              /* server clock */
    double busy_s;             /* time with at least one request running */
} rp_server_stats;

rp_status rp_server_create(const rp_server_config* config, rp_server** out);
void rp_server_destroy(rp_server* server);
/* Deep-copies the request. RP_ERR_BUDGET if it could never fit. */
rp_status rp_server_submit(rp_server* server, const rp_request* request, uint64_t* id);
rp_status rp_server_info(rp_server* server, uint64_t id, rp_request_info* out);
/* Blocks until the request is done; RP_ERR_NOT_READY after timeout_s. */
rp_status rp_server_wait(rp_server* server, uint64_t id, double timeout_s);
/* Final positions of a finished request's rods, xyz floats, rods in request
 * order. RP_ERR_NOT_READY while it runs. */
rp_status rp_server_result(rp_server* server, uint64_t id, float* positions_xyz, int64_t capacity_floats);
/* Forget a finished request (its result memory on the host). */
rp_status rp_server_release(rp_server* server, uint64_t id);
rp_status rp_server_get_stats(rp_server* server, rp_server_stats* out);
/* Blocks until nothing is queued or running; RP_ERR_NOT_READY on timeout. */
rp_status rp_server_drain(rp_server* server, double timeout_s);

/* ---- trajectory files ----
 * reference: the .rodtraj writer of the demo scenes (TrajectoryWriter,
 * src/validation/scenes.cpp:13-20 format, :44-90 writer), fed here from the
 * batch's device buffers without a synchronising download: each append packs
 * the positions on the batch's stream (compensation applied), copies them and
 * the contact states into pinned buffers and returns; a writer thread writes
 * the frame while the next steps run (two frames in flight at most). A frame
 * is the caller's seconds value, every rod's positions (rod-major) and the
 * contact points: the particles of world-contact slots that pushed in the
 * last step. Every rod must have the same particle count (the format's).
 * Close the trajectory before destroying its batch. */
typedef struct rp_traj rp_traj;
rp_status rp_traj_open(const char* path, int32_t num_frames, const rp_batch* batch, float radius, float fps,
                       rp_traj** out);
rp_status rp_traj_append(rp_traj* traj, rp_batch* batch, float seconds);
/* Waits for the queued frames, corrects the header's frame count if fewer or
 * more than declared were appended, closes the file and frees the writer. */
rp_status rp_traj_close(rp_traj* traj, int32_t* frames_written);

#ifdef __cplusplus
}
#endif
#endif /* ROPEPHYSICS_B200_H */
