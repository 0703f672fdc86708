/*
 * rod_oracle.h -- CPU restatement of RopePhysics' XPBD Cosserat-rod step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the GPU path is compared
 * against; nothing in the shipped library links it. Only tests/, the smoke
 * check in __graft_entry__.py and bench.py's CPU-baseline leg load it.
 *
 * It restates, in C++ with a scalar typedef, the reference's FP64 CPU solver and the host-side
 * preprocessing that feeds the GPU batch:
 *   rod model and builders      src/core/rod.h:26-170, src/core/rod.cpp:1-321
 *   greedy constraint colouring src/core/coloring.cpp:11-95
 *   contacts and spatial hash   src/core/collision.h:35-121, collision.cpp:10-152
 *   XPBD substep / step         src/core/solver.h:15-100, solver.cpp:35-290
 *   shared math                 src/core/math3.h:44-353, src/core/geometry.h:17-224
 * The operation order of every floating-point expression follows those files,
 * so the double build reproduces the reference CPU bit for bit (pinned against
 * docs/data/crosscheck.csv and against the reference compiled from source).
 * Compiled with -DORC_FLOAT the same code runs in single precision: the
 * reference's own "float CPU" tie-breaker (src/core/math3.h:15-22). Compiled
 * with -DORC_COUNT the scalar is an op-counting wrapper around double (same
 * memory layout), which gives the exact floating-point operation count of a
 * step -- the numerator of the kernel's FP32-pipe roofline.
 *
 * Memory is owned by the caller: every array in orc_rod is a plain pointer
 * the caller allocated (numpy in the tests).
 */
#ifndef ROD_ORACLE_H
#define ROD_ORACLE_H

#include <stdint.h>

#if defined(ORC_FLOAT)
typedef float orc_real;
#elif defined(ORC_COUNT) && defined(__cplusplus)
#include "orc_counted.h"
typedef orc::Counted orc_real;
#else
typedef double orc_real;
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* One rod, structure of arrays (src/core/rod.h:49-98). Vectors are packed xyz,
 * quaternions packed wxyz. */
typedef struct orc_rod {
    int32_t nP, nS, nSt, nB; /* particles, frames (incl. ghosts), stretch, bend */
    orc_real *x, *xPrev, *v, *invMass, *mass, *extForce, *kinVel; /* nP (x3) */
    orc_real *q, *qPrev, *omega, *invInertia, *inertia, *extTorque; /* nS (x4/x3) */
    int32_t *sP0, *sP1, *sSeg;
    orc_real *sRest, *sComp, *sLam; /* nSt (x3) */
    int32_t *bA, *bB;
    orc_real *bRest, *bRestD, *bComp, *bLam; /* nB (x3) */
    orc_real radius, youngs, poisson, density;
} orc_rod;

/* Colouring (src/core/coloring.h:22-37): `order` holds count entries,
 * `colorStart` numColors + 1 offsets. */
typedef struct orc_coloring {
    int32_t count, numColors;
    int32_t *order;      /* count */
    int32_t *colorStart; /* capacity count + 1 */
} orc_coloring;

/* Primitive (src/core/geometry.h:17-65). */
typedef struct orc_prim {
    int32_t type; /* 0 plane, 1 sphere, 2 capsule, 3 box */
    int32_t pad;
    double a[3], b[3], normal[3], halfExtents[3], rotation[4];
    double radius, friction;
} orc_prim;

/* CollisionWorld (src/core/collision.h:83-106). */
typedef struct orc_world {
    const orc_prim *prims;
    int32_t numPrims;
    int32_t selfCollision;
    double selfFriction;
    int32_t selfSkip;
    int32_t hashTableSize;
    double contactMarginRadii;
} orc_world;

/* Contact (src/core/collision.h:35-48). */
typedef struct orc_contact {
    int32_t idx[4];
    orc_real weight[4];
    orc_real normal[3];
    orc_real offset, friction, lambdaN, appliedTangential;
    int32_t count;
    /* Stick/slip outcome of the last friction pass this contact saw:
     * 0 none (separated or frictionless), 1 stick, 2 slip. Not part of the
     * reference struct; derived from the cap test in projectContacts. */
    int32_t frictionState;
    int32_t prim; /* primitive index (world contacts), -1 for self contacts */
    int32_t pad;
} orc_contact;

/* SolverParams (src/core/solver.h:15-37). */
typedef struct orc_params {
    double dt;
    int32_t substeps, iterations;
    double gravity[3];
    double linearDamping, angularDamping;
    int32_t contactInterval;
    int32_t pad;
    const orc_coloring *stretchColoring; /* NULL = index order */
    const orc_coloring *bendColoring;
} orc_params;

/* Per-rod scratch that persists across steps (src/core/solver.h:41-44). The
 * caller provides contact storage of `capacity` entries. */
typedef struct orc_context {
    orc_contact *contacts;
    int32_t count, capacity;
    int32_t overflow; /* contacts that did not fit `capacity` (never silently lost) */
    int32_t pad;
} orc_context;

/* ---- builders (rod.cpp) ---- */
/* Sizes of a rod built from nPoints centreline points: nP = nPoints,
 * nS = nSt = nPoints - 1, nB = nPoints - 2. Arrays must be allocated by the
 * caller with room for the ghost frame and ghost bend clampEnd adds
 * (nS + 2, nB + 2). */
int orc_build_straight(orc_rod *rod, int32_t numSegments, double length, double youngs,
                       double poisson, double density, double radius, const double origin[3],
                       const double direction[3]);
int orc_build_centerline(orc_rod *rod, const double *points, int32_t numPoints, double youngs,
                         double poisson, double density, double radius,
                         const double frameSeed[3], double twistPerLength);
int32_t orc_clamp_end(orc_rod *rod, int32_t tip); /* returns ghost frame index */
void orc_set_rest_from_current(orc_rod *rod);
void orc_pin_particle(orc_rod *rod, int32_t i);

/* ---- colouring (coloring.cpp) ---- */
void orc_color_stretch(const orc_rod *rod, orc_coloring *out);
void orc_color_bend(const orc_rod *rod, orc_coloring *out);
int32_t orc_self_gap(const orc_rod *rod, const orc_world *world);

/* ---- contacts (collision.cpp) ---- */
void orc_generate_contacts(const orc_rod *rod, const orc_world *world, orc_context *ctx);

/* ---- solver (solver.cpp) ---- */
void orc_step(orc_rod *rod, const orc_params *p);
void orc_step_world(orc_rod *rod, const orc_params *p, const orc_world *world, orc_context *ctx);
/* Many independent rods, contiguous threads over rods (the thread pool of
 * src/gpu/gpu_suite.cpp:88-111, src/validation/scaling_cases.cpp:404-459). */
void orc_step_many(orc_rod *rods, int32_t numRods, const orc_params *p, const orc_world *worlds,
                   const int32_t *worldOfRod, orc_context *ctxs, int32_t steps, int32_t threads);

/* Op counts accumulated since the last reset, by kind: [0] add/sub,
 * [1] mul, [2] div, [3] sqrt, [4] compare, [5] other (floor, exp, trig).
 * All zero unless built with -DORC_COUNT. */
void orc_op_counts(uint64_t out[6]);
void orc_op_reset(void);

#ifdef __cplusplus
}
#endif
#endif
