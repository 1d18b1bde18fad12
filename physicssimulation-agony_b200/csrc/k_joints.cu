// Body constraints: springs, revolute, prismatic and slider joints, motors (Solving/SpringSolver.cpp,
// RevoluteJointSolver.cpp, PrismaticJointSolver.cpp, SliderJointSolver.cpp, MotorSolver.cpp), scheduled as
// ConstraintScheduler::solve does (Solving/ConstraintScheduler.cpp:9-80), between the two integration phases
// (Simulation.cpp:392-407). Paths are relative to PhysicsSimulation-Agony/PS_AGONY2D/.
//
// The reference solves each constraint type's active constraints one after another in dense order (Gauss-Seidel;
// below its threading threshold, one wave in identity order). Here each type's constraints come grouped by level:
// a constraint's level is one more than the highest level of the earlier constraints (in dense order) that write
// one of its bodies. Constraints of one level touch disjoint movable bodies and read only what earlier levels
// wrote, so solving a level in parallel, with a barrier between levels, gives the dense-order results bit for bit.
// One CTA runs the whole schedule: the compute tick over every type, the motors' warm start, then the interleaved
// velocity iterations (type t is active at iteration k when floor((k+1) n_t / max) > floor(k n_t / max)).
//
// Solver data (JointData::s) per kind. Spring: s0, s1 direction, s2 inverse effective mass (0: skip), s3 bias.
// Revolute joint: s0, s1 bias, s4 k11, s5 k12, s6 k22 of the inverse effective mass (all 0: skip). Prismatic and
// slider joints: s0, s1 axis, s2, s3 perpendicular, s4 s1, s5 s2 (perpendicular moment arms), s6 a1, s7 a2 (axis
// moment arms), s8 k11 (slider: the scalar inverse mass, 0: inactive), s9 k12, s10 k22, s11 block valid
// (prismatic), s12 bias1 (slider: bias), s13 bias2, s14 axis inverse effective mass, s15 axis bias, s16 limit
// direction (0: no limit this step), s17 accumulated axis impulse. Motor: s0 inverse inertia (0: skip), s1 inertia,
// s2 target speed, s3 max impulse, s4 impulse.
#include "ag2d_kernels.cuh"

namespace ag2d {

namespace {

constexpr uint32_t K_SPRING = 0, K_REVOLUTE = 1, K_PRISMATIC = 2, K_SLIDER = 3, K_MOTOR = 4;

// glm::clamp for scalars: min(max(x, lo), hi) with max(x, y) = (x < y) ? y : x and min(x, y) = (y < x) ? y : x.
__device__ __forceinline__ float glm_clamp(float x, float lo, float hi)
{
    const float t = (x < lo) ? lo : x;
    return (hi < t) ? hi : t;
}

// Soft-constraint parameters from stiffness and damping (SpringSolver.cpp:92-101 and the same in every joint).
__device__ __forceinline__ void soft_params(float dt, float k, float c, float& gamma, float& beta)
{
    gamma = 0.0f;
    beta = 0.0f;
    const float denom = dt * (c + dt * k);
    if (denom > 1e-12f) {
        gamma = 1.0f / denom;
        beta = dt * k * gamma;
    }
}

// Wraps an angle into (-pi, pi] (PrismaticJointSolver.cpp:12-17).
__device__ __forceinline__ float wrap_to_pi(float angle)
{
    const float pi = 3.14159265358979323846f, twoPi = 2.0f * pi;
    return angle - twoPi * floorf((angle + pi) / twoPi);
}

struct Frame {   // the anchors of a pair constraint in world orientation
    float4 pA, pB;
    float imA, imB;
    float2 cA, cB;
    float rAx, rAy, rBx, rBy;
};
__device__ __forceinline__ Frame frame(const DeviceWorld& w, const JointRec& r)
{
    Frame f;
    f.pA = w.bpos[r.bodyA];
    f.pB = w.bpos[r.bodyB];
    f.imA = w.bvel[r.bodyA].w;
    f.imB = w.bvel[r.bodyB].w;
    f.cA = w.brot[r.bodyA];
    f.cB = w.brot[r.bodyB];
    f.rAx = r.ax * f.cA.x - r.ay * f.cA.y;
    f.rAy = r.ax * f.cA.y + r.ay * f.cA.x;
    f.rBx = r.bx * f.cB.x - r.by * f.cB.y;
    f.rBy = r.bx * f.cB.y + r.by * f.cB.x;
    return f;
}

// computeConstraintData of one spring (SpringSolver.cpp:7-108).
__device__ void spring_data(const DeviceWorld& w, const JointRec& r, float dt, JointData& d)
{
    d.s[2] = 0.0f;
    if (w.bvel[r.bodyA].w == 0.0f && w.bvel[r.bodyB].w == 0.0f) return;
    const Frame f = frame(w, r);
    const float dx = (f.pB.x + f.rBx) - (f.pA.x + f.rAx), dy = (f.pB.y + f.rBy) - (f.pA.y + f.rAy);
    const float lenSq = dx * dx + dy * dy;
    if (lenSq < 1e-12f) return;
    const float len = sqrtf(lenSq);
    const float nx = dx / len, ny = dy / len;
    const float C = len - r.p[0];
    const float raCn = (f.rAx * ny) - (f.rAy * nx);
    const float rbCn = (f.rBx * ny) - (f.rBy * nx);
    const float eff = f.imA + f.imB + f.pA.w * raCn * raCn + f.pB.w * rbCn * rbCn;
    if (eff <= 0.0f) return;
    float gamma, beta;
    soft_params(dt, r.p[1], r.p[2], gamma, beta);
    d.rAx = f.rAx; d.rAy = f.rAy; d.rBx = f.rBx; d.rBy = f.rBy;
    d.s[0] = nx; d.s[1] = ny;
    d.s[2] = 1.0f / (eff + gamma);
    d.s[3] = beta * C;
}

// computeConstraintData of one revolute joint (RevoluteJointSolver.cpp:7-115).
__device__ void revolute_data(const DeviceWorld& w, const JointRec& r, float dt, JointData& d)
{
    d.s[4] = d.s[5] = d.s[6] = 0.0f;
    if (w.bvel[r.bodyA].w == 0.0f && w.bvel[r.bodyB].w == 0.0f) return;
    const Frame f = frame(w, r);
    const float iIA = f.pA.w, iIB = f.pB.w;
    const float ex = (f.pB.x + f.rBx) - (f.pA.x + f.rAx), ey = (f.pB.y + f.rBy) - (f.pA.y + f.rAy);
    const float k11 = f.imA + f.imB + iIA * f.rAy * f.rAy + iIB * f.rBy * f.rBy;
    const float k22 = f.imA + f.imB + iIA * f.rAx * f.rAx + iIB * f.rBx * f.rBx;
    const float k12 = -iIA * f.rAx * f.rAy - iIB * f.rBx * f.rBy;
    float gamma, beta;
    soft_params(dt, r.p[1], r.p[2], gamma, beta);
    const float k11s = k11 + gamma, k22s = k22 + gamma;
    const float det = k11s * k22s - k12 * k12;
    if (det <= 1e-12f) return;
    const float invDet = 1.0f / det;
    d.rAx = f.rAx; d.rAy = f.rAy; d.rBx = f.rBx; d.rBy = f.rBy;
    d.s[0] = beta * ex; d.s[1] = beta * ey;
    d.s[4] = k22s * invDet;
    d.s[6] = k11s * invDet;
    d.s[5] = -k12 * invDet;
}

// computeConstraintData of one prismatic (slider == false; PrismaticJointSolver.cpp:20-158) or slider joint
// (SliderJointSolver.cpp:8-130): the perpendicular (and, prismatic, relative-angle) soft block and the hard
// one-sided axis limit.
__device__ void axis_joint_data(const DeviceWorld& w, const JointRec& r, float dt, bool slider, JointData& d)
{
    d.s[11] = 0.0f;   // block valid (prismatic)
    d.s[8] = 0.0f;    // scalar inverse mass (slider)
    d.s[16] = 0.0f;   // limit direction
    d.s[14] = 0.0f;
    d.s[17] = 0.0f;
    const float invDt = dt > 1e-12f ? 1.0f / dt : 0.0f;
    if (w.bvel[r.bodyA].w == 0.0f && w.bvel[r.bodyB].w == 0.0f) return;
    const Frame f = frame(w, r);
    const float iIA = f.pA.w, iIB = f.pB.w;
    const float dx = (f.pB.x + f.rBx) - (f.pA.x + f.rAx), dy = (f.pB.y + f.rBy) - (f.pA.y + f.rAy);
    const float axX = r.p[0] * f.cA.x - r.p[1] * f.cA.y, axY = r.p[0] * f.cA.y + r.p[1] * f.cA.x;
    const float pX = -axY, pY = axX;
    d.s[0] = axX; d.s[1] = axY; d.s[2] = pX; d.s[3] = pY;
    const float qx = dx + f.rAx, qy = dy + f.rAy;   // d + rotatedAnchorA
    const float s1 = qx * pY - qy * pX, s2 = f.rBx * pY - f.rBy * pX;
    d.s[4] = s1; d.s[5] = s2;
    float gamma, beta;
    soft_params(dt, r.p[2], r.p[3], gamma, beta);
    if (!slider) {
        const float k11 = f.imA + f.imB + iIA * s1 * s1 + iIB * s2 * s2;
        const float k12 = iIA * s1 + iIB * s2;
        float k22 = iIA + iIB;
        if (k22 == 0.0f) k22 = 1.0f;
        const float k11s = k11 + gamma, k22s = k22 + gamma;
        const float det = k11s * k22s - k12 * k12;
        if (det > 1e-12f) {
            const float invDet = 1.0f / det;
            d.s[8] = k22s * invDet;
            d.s[10] = k11s * invDet;
            d.s[9] = -k12 * invDet;
            d.s[11] = 1.0f;
            const float C1 = pX * dx + pY * dy;
            const float rel = wrap_to_pi(f.pB.z - f.pA.z);
            const float C2 = wrap_to_pi(rel - r.p[6]);
            d.s[12] = beta * C1;
            d.s[13] = beta * C2;
        }
    } else {
        const float k = f.imA + f.imB + iIA * s1 * s1 + iIB * s2 * s2;
        const float kSoft = k + gamma;
        if (kSoft > 1e-12f) {
            d.s[8] = 1.0f / kSoft;
            d.s[12] = beta * (pX * dx + pY * dy);
        }
    }
    if (r.flags & 1u) {
        const float translation = axX * dx + axY * dy;
        const float lower = r.p[4], upper = r.p[5];
        float direction = 0.0f, C = 0.0f;
        if (translation <= lower + 0.005f) { direction = 1.0f; C = translation - lower; }
        else if (translation >= upper - 0.005f) { direction = -1.0f; C = translation - upper; }
        if (direction != 0.0f) {
            const float a1 = qx * axY - qy * axX, a2 = f.rBx * axY - f.rBy * axX;
            const float kAxis = f.imA + f.imB + iIA * a1 * a1 + iIB * a2 * a2;
            if (kAxis > 1e-12f) {
                d.s[6] = a1; d.s[7] = a2;
                d.s[14] = 1.0f / kAxis;
                d.s[16] = direction;
                d.s[15] = 0.2f * invDt * C;
            }
        }
    }
}

// computeConstraintData of one motor (MotorSolver.cpp:7-45); the clamped accumulated impulse is written back.
__device__ void motor_data(const DeviceWorld& w, const JointRec& r, float dt, float* impulses, JointData& d)
{
    const float iI = w.bpos[r.bodyA].w;
    d.s[0] = iI;
    if (iI == 0.0f) {
        impulses[r.index] = 0.0f;
        return;
    }
    const float maxImpulse = r.p[1] * dt;
    const float impulse = glm_clamp(impulses[r.index], -maxImpulse, maxImpulse);
    d.s[1] = 1.0f / iI;
    d.s[2] = r.p[0];
    d.s[3] = maxImpulse;
    d.s[4] = impulse;
    impulses[r.index] = impulse;
}

// Applies a point impulse to both bodies, as the spring and revolute solvers do (A gains, B loses).
__device__ __forceinline__ void apply_pair(const DeviceWorld& w, uint32_t a, uint32_t b, float4 vA, float4 vB,
                                           float iIA, float iIB, const JointData& d, float ix, float iy)
{
    if (vA.w > 0.0f) {
        vA.x = vA.x + ix * vA.w;
        vA.y = vA.y + iy * vA.w;
        const float tA = d.rAx * iy - d.rAy * ix;
        vA.z = vA.z + tA * iIA;
        w.bvel[a] = vA;
    }
    if (vB.w > 0.0f) {
        vB.x = vB.x - ix * vB.w;
        vB.y = vB.y - iy * vB.w;
        const float tB = d.rBx * iy - d.rBy * ix;
        vB.z = vB.z - tB * iIB;
        w.bvel[b] = vB;
    }
}

// Relative velocity of the anchors, B's minus A's (SpringSolver.cpp:140-147).
__device__ __forceinline__ float2 anchor_relative_velocity(float4 vA, float4 vB, const JointData& d)
{
    const float aAx = (-d.rAy) * vA.z, aAy = d.rAx * vA.z;
    const float aBx = (-d.rBy) * vB.z, aBy = d.rBx * vB.z;
    return make_float2((vB.x + aBx) - (vA.x + aAx), (vB.y + aBy) - (vA.y + aAy));
}

__device__ void spring_solve(const DeviceWorld& w, const JointRec& r, const JointData& d)
{
    if (d.s[2] == 0.0f) return;
    const float4 vA = w.bvel[r.bodyA], vB = w.bvel[r.bodyB];
    const float iIA = w.bpos[r.bodyA].w, iIB = w.bpos[r.bodyB].w;
    const float2 rv = anchor_relative_velocity(vA, vB, d);
    const float cdot = rv.x * d.s[0] + rv.y * d.s[1];
    const float mag = (cdot + d.s[3]) * d.s[2];
    apply_pair(w, r.bodyA, r.bodyB, vA, vB, iIA, iIB, d, d.s[0] * mag, d.s[1] * mag);
}

__device__ void revolute_solve(const DeviceWorld& w, const JointRec& r, const JointData& d)
{
    if (d.s[4] == 0.0f && d.s[5] == 0.0f && d.s[6] == 0.0f) return;
    const float4 vA = w.bvel[r.bodyA], vB = w.bvel[r.bodyB];
    const float iIA = w.bpos[r.bodyA].w, iIB = w.bpos[r.bodyB].w;
    const float2 rv = anchor_relative_velocity(vA, vB, d);
    const float hx = rv.x + d.s[0], hy = rv.y + d.s[1];
    const float ix = d.s[4] * hx + d.s[5] * hy;
    const float iy = d.s[5] * hx + d.s[6] * hy;
    apply_pair(w, r.bodyA, r.bodyB, vA, vB, iIA, iIB, d, ix, iy);
}

// One velocity iteration of a prismatic (PrismaticJointSolver.cpp:160-255) or slider joint (SliderJointSolver.cpp:
// 132-220): the perpendicular block, then the axis limit with its accumulated, one-sided impulse.
__device__ void axis_joint_solve(const DeviceWorld& w, const JointRec& r, JointData& d, bool slider)
{
    const bool block = slider ? d.s[8] > 0.0f : d.s[11] != 0.0f;
    if (!block && d.s[16] == 0.0f) return;
    float4 vA = w.bvel[r.bodyA], vB = w.bvel[r.bodyB];
    const float imA = vA.w, imB = vB.w;
    const float iIA = w.bpos[r.bodyA].w, iIB = w.bpos[r.bodyB].w;
    if (block) {
        const float pX = d.s[2], pY = d.s[3], s1 = d.s[4], s2 = d.s[5];
        const float cdot1 = (pX * (vB.x - vA.x) + pY * (vB.y - vA.y)) + s2 * vB.z - s1 * vA.z;
        float l1, LA, LB;
        if (slider) {
            l1 = -d.s[8] * (cdot1 + d.s[12]);
            LA = l1 * s1;
            LB = l1 * s2;
        } else {
            const float cdot2 = vB.z - vA.z;
            const float rhs1 = cdot1 + d.s[12], rhs2 = cdot2 + d.s[13];
            l1 = -(d.s[8] * rhs1 + d.s[9] * rhs2);
            const float l2 = -(d.s[9] * rhs1 + d.s[10] * rhs2);
            LA = l1 * s1 + l2;
            LB = l1 * s2 + l2;
        }
        const float Px = pX * l1, Py = pY * l1;
        vA.x = vA.x - Px * imA; vA.y = vA.y - Py * imA;
        vA.z = vA.z - LA * iIA;
        vB.x = vB.x + Px * imB; vB.y = vB.y + Py * imB;
        vB.z = vB.z + LB * iIB;
    }
    if (d.s[16] != 0.0f) {
        const float axX = d.s[0], axY = d.s[1], a1 = d.s[6], a2 = d.s[7];
        const float cdot = (axX * (vB.x - vA.x) + axY * (vB.y - vA.y)) + a2 * vB.z - a1 * vA.z;
        const float raw = -(cdot + d.s[15]) * d.s[14];
        const float oldImpulse = d.s[17];
        const float sum = oldImpulse + raw;
        const float newImpulse = d.s[16] > 0.0f ? (sum < 0.0f ? 0.0f : sum) : (0.0f < sum ? 0.0f : sum);
        const float applied = newImpulse - oldImpulse;
        d.s[17] = newImpulse;
        const float Px = axX * applied, Py = axY * applied;
        const float LA = applied * a1, LB = applied * a2;
        vA.x = vA.x - Px * imA; vA.y = vA.y - Py * imA;
        vA.z = vA.z - LA * iIA;
        vB.x = vB.x + Px * imB; vB.y = vB.y + Py * imB;
        vB.z = vB.z + LB * iIB;
    }
    if (imA > 0.0f) w.bvel[r.bodyA] = vA;
    if (imB > 0.0f) w.bvel[r.bodyB] = vB;
}

__device__ void motor_warm(const DeviceWorld& w, const JointRec& r, const JointData& d)
{
    if (d.s[0] == 0.0f) return;
    float4 v = w.bvel[r.bodyA];
    v.z = v.z + d.s[4] * d.s[0];
    w.bvel[r.bodyA] = v;
}

__device__ void motor_solve(const DeviceWorld& w, const JointRec& r, JointData& d, float* impulses)
{
    if (d.s[0] == 0.0f) return;
    float4 v = w.bvel[r.bodyA];
    const float lambda = (d.s[2] - v.z) * d.s[1];
    const float oldImpulse = d.s[4];
    const float newImpulse = glm_clamp(oldImpulse + lambda, -d.s[3], d.s[3]);
    d.s[4] = newImpulse;
    impulses[r.index] = newImpulse;
    v.z = v.z + (newImpulse - oldImpulse) * d.s[0];
    w.bvel[r.bodyA] = v;
}

__device__ __forceinline__ void solve_one(const DeviceWorld& w, uint32_t k, const JointRec& r, JointData& d,
                                          float* impulses)
{
    switch (k) {
    case K_SPRING: spring_solve(w, r, d); break;
    case K_REVOLUTE: revolute_solve(w, r, d); break;
    case K_PRISMATIC: axis_joint_solve(w, r, d, false); break;
    case K_SLIDER: axis_joint_solve(w, r, d, true); break;
    default: motor_solve(w, r, d, impulses); break;
    }
}

}  // namespace

__global__ void __launch_bounds__(JOINT_THREADS) k_joints(DeviceWorld w, JointLaunch L)
{
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    // Compute tick: every type's constraint data, read-only on the bodies.
    for (uint32_t k = 0; k < JOINT_KINDS_DEVICE; k++)
        for (uint32_t i = tid; i < L.count[k]; i += nt) {
            JointData d;
            const JointRec r = L.rec[k][i];
            switch (k) {
            case K_SPRING: spring_data(w, r, L.dt, d); break;
            case K_REVOLUTE: revolute_data(w, r, L.dt, d); break;
            case K_PRISMATIC: axis_joint_data(w, r, L.dt, false, d); break;
            case K_SLIDER: axis_joint_data(w, r, L.dt, true, d); break;
            default: motor_data(w, r, L.dt, L.motorImpulse, d); break;
            }
            L.data[k][i] = d;
        }
    __syncthreads();
    // Warm start: the motors (the one type with a warm start), level by level.
    for (uint32_t l = 0; l < L.levels[K_MOTOR]; l++) {
        for (uint32_t i = L.levelStart[K_MOTOR][l] + tid; i < L.levelStart[K_MOTOR][l + 1]; i += nt)
            motor_warm(w, L.rec[K_MOTOR][i], L.data[K_MOTOR][i]);
        __syncthreads();
    }
    // Velocity iterations, the types interleaved in ConstraintType order.
    for (uint32_t it = 0; it < L.maxIterations; it++)
        for (uint32_t k = 0; k < JOINT_KINDS_DEVICE; k++) {
            const uint64_t n = L.iterations[k];
            if (L.count[k] == 0 || (uint64_t(it + 1) * n) / L.maxIterations == (uint64_t(it) * n) / L.maxIterations)
                continue;
            for (uint32_t l = 0; l < L.levels[k]; l++) {
                for (uint32_t i = L.levelStart[k][l] + tid; i < L.levelStart[k][l + 1]; i += nt)
                    solve_one(w, k, L.rec[k][i], L.data[k][i], L.motorImpulse);
                __syncthreads();
            }
        }
}

}  // namespace ag2d
