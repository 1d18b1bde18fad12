/* CPU restatement of PS_AGONY2D's per-step collision and contact pipeline.
 *
 * TEST INFRASTRUCTURE (the oracle). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and only as the checker. The product path never calls it.
 *
 * Every function restates one reference function in plain C with the reference's fp32 operation order
 * (no FMA contraction; explicit fmaf only where the reference's SIMD code issues an FMA instruction). Each
 * definition in ag2d_oracle.c cites the reference file and lines it follows (paths relative to
 * PhysicsSimulation-Agony/PS_AGONY2D/).
 *
 * Parity is pinned against the reference itself: tests/golden/ holds vectors produced by the reference engine
 * compiled on the CPU (oracle/ref_build.sh, tests/golden/make_golden.py).
 */
#ifndef AG2D_ORACLE_H
#define AG2D_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORA_CIRCLE = 0, ORA_BOX = 1, ORA_POLYGON = 2 };
enum { ORA_STATIC = 0, ORA_SLEEPING = 1, ORA_DYNAMIC = 2 };

/* One world in the reference's dense layout. Group starts follow GroupRanges (GroupRanges.h:130-157):
 * group g occupies [starts[g], starts[g+1]) for g in {static, sleeping, dynamic}; starts[3] is the live count. */
typedef struct ora_world {
    uint32_t n_bodies, n_colliders, n_materials;
    uint32_t body_starts[4];
    uint32_t col_starts[4];
    /* bodies */
    float *comX, *comY, *velX, *velY, *rot, *angVel, *invMass, *invInertia, *rotCos, *rotSin;
    float *wrapCount, *boundRadius, *sleepTimer;
    uint32_t *islandId;
    /* colliders */
    uint32_t *bodyIndex, *shapeType, *shapeIndex, *material;
    float *comOffX, *comOffY, *localRot;
    float *worldX, *worldY, *worldRot, *worldCos, *worldSin;
    float *minX, *minY, *maxX, *maxY;
    /* shapes, indexed by shapeIndex of their type */
    float *circleRadius;
    float *boxHalfW, *boxHalfH;
    uint32_t *polyOffset, *polyCount; /* into polyVerts / polyNormals (float2 each) */
    float *polyVerts, *polyNormals;
    /* materials */
    float *matElasticity, *matStaticFriction, *matDynamicFriction;
} ora_world;

typedef struct ora_manifold {
    uint32_t a, b;           /* dense collider indices (A = reference collider of the normal's origin) */
    float nx, ny, depth;
    uint32_t count;
    float px[2], py[2];
    uint32_t id[2];
    float jn[2], jt[2];      /* persistent normal / tangent impulse accumulators */
} ora_manifold;

/* ---- integration, wrap, rotation cos/sin ---- */
void ora_integrate_velocity_verlet(ora_world *w, uint32_t begin, uint32_t end, float dt, float gx, float gy,
                                   float angular_damping);
void ora_wrap_body_rotations(ora_world *w, uint32_t begin, uint32_t end);
void ora_fastcossin_array(const float *in, float *out_cos, float *out_sin, uint32_t n);
void ora_body_cossin(ora_world *w, uint32_t begin, uint32_t end);

/* ---- collider poses and AABBs ---- */
void ora_collider_world_positions(ora_world *w, uint32_t begin, uint32_t end);
void ora_collider_world_rotations(ora_world *w, uint32_t begin, uint32_t end);
void ora_collider_aabbs(ora_world *w, uint32_t begin, uint32_t end);

/* ---- Morton keys and the stable key sort of one tree's collider range ---- */
void ora_morton_codes(const ora_world *w, uint32_t begin, uint32_t end, uint32_t *out_codes, float *out_bounds4);
void ora_sort_by_morton(const uint32_t *codes, uint32_t begin, uint32_t n, uint32_t *out_sorted_colliders,
                        uint32_t *out_sorted_codes);

/* ---- broad phase: the canonical candidate pair set ----
 * Writes pairs as (a, b) with a dynamic; dynamic-dynamic pairs have a < b (dense index) in this canonical form.
 * Returns the number of pairs, or -(needed) if cap is too small. */
int64_t ora_broad_pairs(const ora_world *w, uint32_t *out_pairs, int64_t cap);

/* ---- narrow phase ----
 * Orients each pair like NarrowPhaseCollisionDetector::processPairs and runs the shape-pair method; writes one
 * manifold per colliding pair (in pair order) and returns how many. */
int64_t ora_narrow(const ora_world *w, const uint32_t *pairs, int64_t n_pairs, ora_manifold *out);

/* Warm start: copies persistent impulses from prev (previous step, collider keys given by prev_slot*) into cur
 * (keys cur_slot*), following finalizeResults/rebuildContactCache. */
void ora_warm_start(const ora_manifold *prev, const uint32_t *prev_slotA, const uint32_t *prev_slotB, int64_t n_prev,
                    ora_manifold *cur, const uint32_t *cur_slotA, const uint32_t *cur_slotB, int64_t n_cur);

/* ---- contact solver (sequential impulses) in a given constraint order ----
 * order[c] selects the manifold solved c-th (NULL = 0..n-1). Updates body velocities/positions and the manifold
 * impulses. The _f64 variant performs every operation in double precision (the replay reference). */
void ora_solve(ora_world *w, ora_manifold *m, int64_t n, const int64_t *order, uint32_t vel_iters,
               uint32_t pos_iters);
void ora_solve_f64(ora_world *w, ora_manifold *m, int64_t n, const int64_t *order, uint32_t vel_iters,
                   uint32_t pos_iters, double *io_vel /* 3 per body: vx, vy, w */, double *io_pos /* 2 per body */,
                   double *out_impulses /* 4 per manifold */);

/* ---- collision events (BodyCollisionSolver::computeConstraintData, Solving/BodyCollisionSolver.cpp:320-387) ----
 * For each manifold in list order, the impact impulse from the world's current velocities (the largest over the
 * contact points of the approach speed along the normal times the normal effective mass, from 0 by std::fmax); a
 * side fires when its collider's callback id is not 0, the impulse is positive and it reaches the collider's
 * threshold. Side a's event comes before side b's. Returns the number of events, or -(needed) if cap is too small. */
typedef struct ora_event {
    uint32_t self, other, selfBody, otherBody, callback;
    float px, py, nx, ny, impulse;
} ora_event;
int64_t ora_collision_events(const ora_world *w, const ora_manifold *m, int64_t n, const uint32_t *callback,
                             const float *threshold, ora_event *out, int64_t cap);

/* ---- islands and sleep flags ----
 * Island ids for dynamic bodies from body-pair edges (ids ordered by DSU root, IslandManager.cpp:36-80), then the
 * sleep-timer update and the per-island "all quiet long enough" AND (ObjectManager.cpp:1438-1491).
 * out_sleep[i] = 1 for each dynamic body that falls asleep this step. Returns the island count. */
uint32_t ora_islands(const ora_world *w, const uint32_t *edges, int64_t n_edges, uint32_t *out_island_id);
void ora_update_sleeping(ora_world *w, const uint32_t *island_id, uint32_t island_count, float dt,
                         float speed_threshold, float time_threshold, uint8_t *out_sleep);

#ifdef __cplusplus
}
#endif
#endif
