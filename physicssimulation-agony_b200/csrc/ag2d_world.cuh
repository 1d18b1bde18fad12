// Device-resident world state (HBM layout) and small device utilities shared by the kernels.
//
// Layout: structure of arrays, with the fields the solver gathers per body packed into float4 so one 16-byte load
// serves a contact end: bvel = (vx, vy, w, invMass), bpos = (x, y, rotation, invInertia). Colliders keep their
// world pose in one float4 (x, y, cos, sin) and their AABB in another (minX, minY, maxX, maxY).
//
// Collider and body indices follow the reference's dense order (GroupRanges.h: static, sleeping, dynamic at
// creation); sleeping is a per-body state flag here instead of a dense-range move, and the per-step work lists
// (dynamic bodies, dynamic colliders, static+sleeping colliders) are compacted index lists rebuilt on state changes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ag2d {

// STATE_DESTROYED: a body removed by a destroy command; it keeps its slot but is in no work list or tree.
enum BodyState : uint8_t { STATE_STATIC = 0, STATE_SLEEPING = 1, STATE_DYNAMIC = 2, STATE_DESTROYED = 3 };

// Error bits of the per-step status word (a device-side failure never traps; the host reads this word).
enum StatusBits : uint32_t {
    STATUS_PAIR_OVERFLOW = 1u << 0,
    STATUS_MANIFOLD_OVERFLOW = 1u << 1,
    STATUS_BARRIER_TIMEOUT = 1u << 2,
    STATUS_LOOKBACK_TIMEOUT = 1u << 3,
    STATUS_COLOR_OVERFLOW = 1u << 4,
    STATUS_HASH_FULL = 1u << 5,
    STATUS_STACK_OVERFLOW = 1u << 6,
    STATUS_EVENT_OVERFLOW = 1u << 7,
};

// Counters written by the kernels and read back by the host after each step (one 64-byte transfer).
struct StepCounters {
    uint32_t status;          // StatusBits
    uint32_t pairs;           // broad-phase candidate pairs
    uint32_t manifolds;       // narrow-phase manifolds (>= 1 contact)
    uint32_t colors;          // solver colours used
    uint32_t woke;            // bodies woken this step
    uint32_t slept;           // bodies put to sleep this step
    uint32_t topoDirty;       // a body changed state: rebuild work lists before the next step
    uint32_t warmHits;        // manifolds that took warm-start impulses
    uint32_t barrierRounds;   // colouring rounds
    uint32_t ccdHits;         // bodies moved back by continuous collision detection
    uint32_t restored;        // sleeping-island manifolds that joined this step's list whole
    uint32_t stored;          // sleeping-island manifolds held when the step began
    uint32_t staged;          // of which the woken islands' records taken out by this step's restore
    uint32_t events;          // collision events recorded (may exceed the event ring: STATUS_EVENT_OVERFLOW)
    uint32_t pad[2];
};

// Manifold record (64 bytes), NarrowPhaseCollisionDetector.h:26-61 minus the handle union: colliders are stable
// device indices. Collider a is the reference side of the normal (normal points from a to b).
struct alignas(16) Manifold {
    uint32_t a, b;
    float nx, ny;
    float depth;
    uint32_t count;
    uint32_t id0, id1;
    float px0, py0, px1, py1;
    float jn0, jt0, jn1, jt1;     // persistent impulse accumulators (warm start)
};
static_assert(sizeof(Manifold) == 64, "Manifold is 64 bytes");

// Collision event (48 bytes), one per opted-in collider side of a manifold: the fields of the reference's
// CollisionEvent (Types/CollisionEvent.h:18-26) with dense indices for the handles, plus the manifold it came from
// and the side (0: self is the manifold's collider a) so the host can put the events in manifold order.
struct alignas(16) EventRecord {
    uint32_t manifold, side, self, other;
    uint32_t selfBody, otherBody, callback;
    float impulse;          // impact impulse: max over the points of approach speed x normal effective mass
    float px, py, nx, ny;   // average of the contact points; the normal from self towards other
};
static_assert(sizeof(EventRecord) == 48, "EventRecord is 48 bytes");

// Collider opt-in for collision events: callback id (0: none) and the impulse threshold.
struct ColliderEvent {
    uint32_t callback;
    float threshold;
};

// Body constraint on the device (SoA/Constraints/*), one per active constraint in solving order: bodies, the
// constraint's dense index in its system, flags (bit 0: the axis limit is enabled), local anchors and parameters.
// Spring: p0 rest length, p1 stiffness, p2 damping. Revolute joint: p1 stiffness, p2 damping. Prismatic and slider
// joints: p0, p1 the local axis of body A (unit), p2 stiffness, p3 damping, p4 lower limit, p5 upper limit,
// p6 reference angle (prismatic). Motor: p0 target speed, p1 max torque.
struct alignas(16) JointRec {
    uint32_t bodyA, bodyB, index, flags;
    float ax, ay, bx, by;
    float p[8];
};
static_assert(sizeof(JointRec) == 64, "JointRec is 64 bytes");

// Per-constraint solver data (the solvers' ConstraintData, Solving/*Solver.h): rotated anchors, then per kind
// the fields listed beside the kernel that fills them (k_joints.cu).
struct alignas(16) JointData {
    float rAx, rAy, rBx, rBy;
    float s[20];
};
static_assert(sizeof(JointData) == 96, "JointData is 96 bytes");

// Per-constraint solver record (128 bytes), built from a Manifold in solving (colour) order: the fields of
// BodyCollisionSolver's VelocityHotData, PositionHotData, VelocityConstraintData and FrictionData.
struct alignas(16) Constraint {
    uint32_t bodyA, bodyB, count, manifold;
    float nx, ny, imA, imB;
    float iIA, iIB, sf, df;
    float jn0, jt0, jn1, jt1;
    float rAn0, rBn0, rAt0, rBt0;
    float nm0, tm0, bias0, penBase;
    float rAn1, rBn1, rAt1, rBt1;
    float nm1, tm1, bias1, pad;
};
static_assert(sizeof(Constraint) == 128, "Constraint is 128 bytes");

struct DeviceWorld {
    uint32_t nBodies, nColliders, nMaterials;
    // Bodies.
    float4* bvel;          // vx, vy, w, invMass
    float4* bpos;          // x, y, rotation, invInertia
    float2* brot;          // rotation cos, sin
    float* wrapCount;      // renderRotationWrapCount
    float* boundRadius;
    float* sleepTimer;
    uint8_t* bstate;       // BodyState
    uint32_t* sleepIsland; // island id while sleeping (the island's root body index)
    // Colliders.
    uint32_t* cbody;       // owner body
    uint32_t* cshape;      // type << 30 | shape index
    uint32_t* cmat;        // material index
    float4* coff;          // comOffsetX, comOffsetY, localRotation, 0
    float4* cpose;         // world x, y, cos, sin
    float* cworldRot;      // wrapped world rotation
    float4* caabb;         // minX, minY, maxX, maxY
    // Shapes.
    float* circleRadius;
    float2* boxHalf;       // boxes: halfWidth, halfHeight; capsules (the same table): halfLength, radius
    uint32_t* polyOffset;  // into polyVerts / polyNormals
    uint32_t* polyCount;
    float2* polyVerts;
    float2* polyNormals;
    // Materials: elasticity, static friction, dynamic friction.
    float4* materials;
    // World partition of a batch (null for a single world): world of each body / collider and the first body /
    // collider of each world ([nWorlds + 1]).
    uint32_t nWorlds;
    uint32_t* bodyWorld;
    uint32_t* colWorld;
    uint32_t* worldBodyStart;
    uint32_t* worldColStart;
    uint32_t* worldDirty;   // set when a body of the world woke or fell asleep this step
};

__host__ __device__ __forceinline__ uint32_t shape_type(uint32_t packed) { return packed >> 30; }
__host__ __device__ __forceinline__ uint32_t shape_index(uint32_t packed) { return packed & 0x3FFFFFFFu; }

// Order-preserving float <-> uint32 map for atomicMin/atomicMax on floats.
__device__ __forceinline__ uint32_t float_to_ordered(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ordered_to_float(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Spin-wait budget for inter-CTA waits (decoupled look-back, grid barriers). A wait that exhausts it records a
// status bit and gives up instead of hanging the GPU.
constexpr uint32_t SPIN_LIMIT = 1u << 22;

// Grid-wide barrier for cooperative launches (all CTAs co-resident). 'bar' is {arrive count, generation}, zeroed
// before launch. Returns false (and sets STATUS_BARRIER_TIMEOUT) if the wait ran out.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t* status)
{
    __syncthreads();
    __shared__ int ok;
    if (threadIdx.x == 0) {
        ok = 1;
        volatile uint32_t* gen = bar + 1;
        const uint32_t g = *gen;
        __threadfence();
        const uint32_t arrived = atomicAdd(bar, 1u);
        if (arrived == gridDim.x - 1) {
            bar[0] = 0;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g) {
                if (++spins > SPIN_LIMIT) { atomicOr(status, STATUS_BARRIER_TIMEOUT); ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0 && (*(volatile uint32_t*)status & STATUS_BARRIER_TIMEOUT) == 0;
}

}  // namespace ag2d
