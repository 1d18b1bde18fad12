// Body constraints: springs, revolute joints and motors (Solving/SpringSolver.cpp, RevoluteJointSolver.cpp,
// MotorSolver.cpp), scheduled as ConstraintScheduler::solve does (Solving/ConstraintScheduler.cpp:9-80), between the
// two integration phases (Simulation.cpp:392-407). Paths are relative to PhysicsSimulation-Agony/PS_AGONY2D/.
//
// The reference solves each constraint type's active constraints one after another in dense order (Gauss-Seidel;
// below its threading threshold, one wave in identity order). Here each type's constraints come grouped by level:
// a constraint's level is one more than the highest level of the earlier constraints (in dense order) that write
// one of its bodies. Constraints of one level touch disjoint movable bodies and read only what earlier levels
// wrote, so solving a level in parallel, with a barrier between levels, gives the dense-order results bit for bit.
// One CTA runs the whole schedule: the compute tick over every type, the motors' warm start, then the interleaved
// velocity iterations (type t is active at iteration k when floor((k+1) n_t / max) > floor(k n_t / max)).
#include "ag2d_kernels.cuh"

namespace ag2d {

namespace {

// glm::clamp for scalars: min(max(x, lo), hi) with max(x, y) = (x < y) ? y : x and min(x, y) = (y < x) ? y : x.
__device__ __forceinline__ float glm_clamp(float x, float lo, float hi)
{
    const float t = (x < lo) ? lo : x;
    return (hi < t) ? hi : t;
}

// Soft-constraint parameters from stiffness and damping (SpringSolver.cpp:92-101, RevoluteJointSolver.cpp:88-97).
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

// computeConstraintData of one spring (SpringSolver.cpp:7-108).
__device__ void spring_data(const DeviceWorld& w, const JointRec& r, float dt, JointData& d)
{
    d.s2 = 0.0f;   // inverse effective mass: 0 skips the spring
    const float4 pA = w.bpos[r.bodyA], pB = w.bpos[r.bodyB];
    const float imA = w.bvel[r.bodyA].w, imB = w.bvel[r.bodyB].w;
    if (imA == 0.0f && imB == 0.0f) return;
    const float2 cA = w.brot[r.bodyA], cB = w.brot[r.bodyB];
    const float rAx = r.ax * cA.x - r.ay * cA.y, rAy = r.ax * cA.y + r.ay * cA.x;
    const float rBx = r.bx * cB.x - r.by * cB.y, rBy = r.bx * cB.y + r.by * cB.x;
    const float dx = (pB.x + rBx) - (pA.x + rAx), dy = (pB.y + rBy) - (pA.y + rAy);
    const float lenSq = dx * dx + dy * dy;
    if (lenSq < 1e-12f) return;
    const float len = sqrtf(lenSq);
    const float nx = dx / len, ny = dy / len;
    const float C = len - r.p0;
    const float raCn = (rAx * ny) - (rAy * nx);
    const float rbCn = (rBx * ny) - (rBy * nx);
    const float eff = imA + imB + pA.w * raCn * raCn + pB.w * rbCn * rbCn;
    if (eff <= 0.0f) return;
    float gamma, beta;
    soft_params(dt, r.p1, r.p2, gamma, beta);
    d.rAx = rAx; d.rAy = rAy; d.rBx = rBx; d.rBy = rBy;
    d.s0 = nx; d.s1 = ny;
    d.s2 = 1.0f / (eff + gamma);
    d.s3 = beta * C;
}

// computeConstraintData of one revolute joint (RevoluteJointSolver.cpp:7-115).
__device__ void revolute_data(const DeviceWorld& w, const JointRec& r, float dt, JointData& d)
{
    d.s4 = d.s5 = d.s6 = 0.0f;   // inverse effective mass matrix: all 0 skips the joint
    const float4 pA = w.bpos[r.bodyA], pB = w.bpos[r.bodyB];
    const float imA = w.bvel[r.bodyA].w, imB = w.bvel[r.bodyB].w;
    if (imA == 0.0f && imB == 0.0f) return;
    const float iIA = pA.w, iIB = pB.w;
    const float2 cA = w.brot[r.bodyA], cB = w.brot[r.bodyB];
    const float rAx = r.ax * cA.x - r.ay * cA.y, rAy = r.ax * cA.y + r.ay * cA.x;
    const float rBx = r.bx * cB.x - r.by * cB.y, rBy = r.bx * cB.y + r.by * cB.x;
    const float ex = (pB.x + rBx) - (pA.x + rAx), ey = (pB.y + rBy) - (pA.y + rAy);
    const float k11 = imA + imB + iIA * rAy * rAy + iIB * rBy * rBy;
    const float k22 = imA + imB + iIA * rAx * rAx + iIB * rBx * rBx;
    const float k12 = -iIA * rAx * rAy - iIB * rBx * rBy;
    float gamma, beta;
    soft_params(dt, r.p1, r.p2, gamma, beta);
    const float k11s = k11 + gamma, k22s = k22 + gamma;
    const float det = k11s * k22s - k12 * k12;
    if (det <= 1e-12f) return;
    const float invDet = 1.0f / det;
    d.rAx = rAx; d.rAy = rAy; d.rBx = rBx; d.rBy = rBy;
    d.s0 = beta * ex; d.s1 = beta * ey;
    d.s4 = k22s * invDet;
    d.s6 = k11s * invDet;
    d.s5 = -k12 * invDet;
}

// computeConstraintData of one motor (MotorSolver.cpp:7-45); the clamped accumulated impulse is written back.
__device__ void motor_data(const DeviceWorld& w, const JointRec& r, float dt, float* impulses, JointData& d)
{
    const float iI = w.bpos[r.bodyA].w;
    d.s0 = iI;
    if (iI == 0.0f) {
        impulses[r.index] = 0.0f;
        return;
    }
    const float maxImpulse = r.p1 * dt;
    const float impulse = glm_clamp(impulses[r.index], -maxImpulse, maxImpulse);
    d.s1 = 1.0f / iI;
    d.s2 = r.p0;
    d.s3 = maxImpulse;
    d.s4 = impulse;
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
    if (d.s2 == 0.0f) return;
    const float4 vA = w.bvel[r.bodyA], vB = w.bvel[r.bodyB];
    const float iIA = w.bpos[r.bodyA].w, iIB = w.bpos[r.bodyB].w;
    const float2 rv = anchor_relative_velocity(vA, vB, d);
    const float cdot = rv.x * d.s0 + rv.y * d.s1;
    const float mag = (cdot + d.s3) * d.s2;
    apply_pair(w, r.bodyA, r.bodyB, vA, vB, iIA, iIB, d, d.s0 * mag, d.s1 * mag);
}

__device__ void revolute_solve(const DeviceWorld& w, const JointRec& r, const JointData& d)
{
    if (d.s4 == 0.0f && d.s5 == 0.0f && d.s6 == 0.0f) return;
    const float4 vA = w.bvel[r.bodyA], vB = w.bvel[r.bodyB];
    const float iIA = w.bpos[r.bodyA].w, iIB = w.bpos[r.bodyB].w;
    const float2 rv = anchor_relative_velocity(vA, vB, d);
    const float hx = rv.x + d.s0, hy = rv.y + d.s1;
    const float ix = d.s4 * hx + d.s5 * hy;
    const float iy = d.s5 * hx + d.s6 * hy;
    apply_pair(w, r.bodyA, r.bodyB, vA, vB, iIA, iIB, d, ix, iy);
}

__device__ void motor_warm(const DeviceWorld& w, const JointRec& r, const JointData& d)
{
    if (d.s0 == 0.0f) return;
    float4 v = w.bvel[r.bodyA];
    v.z = v.z + d.s4 * d.s0;
    w.bvel[r.bodyA] = v;
}

__device__ void motor_solve(const DeviceWorld& w, const JointRec& r, JointData& d, float* impulses)
{
    if (d.s0 == 0.0f) return;
    float4 v = w.bvel[r.bodyA];
    const float lambda = (d.s2 - v.z) * d.s1;
    const float oldImpulse = d.s4;
    const float newImpulse = glm_clamp(oldImpulse + lambda, -d.s3, d.s3);
    d.s4 = newImpulse;
    impulses[r.index] = newImpulse;
    v.z = v.z + (newImpulse - oldImpulse) * d.s0;
    w.bvel[r.bodyA] = v;
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
            if (k == 0) spring_data(w, r, L.dt, d);
            else if (k == 1) revolute_data(w, r, L.dt, d);
            else motor_data(w, r, L.dt, L.motorImpulse, d);
            L.data[k][i] = d;
        }
    __syncthreads();
    // Warm start: the motors, level by level.
    for (uint32_t l = 0; l < L.levels[2]; l++) {
        for (uint32_t i = L.levelStart[2][l] + tid; i < L.levelStart[2][l + 1]; i += nt)
            motor_warm(w, L.rec[2][i], L.data[2][i]);
        __syncthreads();
    }
    // Velocity iterations, the types interleaved.
    for (uint32_t it = 0; it < L.maxIterations; it++)
        for (uint32_t k = 0; k < JOINT_KINDS_DEVICE; k++) {
            const uint64_t n = L.iterations[k];
            if (L.count[k] == 0 || (uint64_t(it + 1) * n) / L.maxIterations == (uint64_t(it) * n) / L.maxIterations)
                continue;
            for (uint32_t l = 0; l < L.levels[k]; l++) {
                for (uint32_t i = L.levelStart[k][l] + tid; i < L.levelStart[k][l + 1]; i += nt) {
                    const JointRec r = L.rec[k][i];
                    if (k == 0) spring_solve(w, r, L.data[0][i]);
                    else if (k == 1) revolute_solve(w, r, L.data[1][i]);
                    else motor_solve(w, r, L.data[2][i], L.motorImpulse);
                }
                __syncthreads();
            }
        }
}

}  // namespace ag2d
