// Collision events: the event records of BodyCollisionSolver::computeConstraintData
// (PhysicsSimulation-Agony/PS_AGONY2D/Solving/BodyCollisionSolver.cpp:320-387) as a device ring.
//
// The reference computes, beside each manifold's constraint data, the impact impulse (the largest over the contact
// points of approach speed along the normal times the normal effective mass, before warm starting) and appends an
// event for each side whose collider has a callback and a threshold the impulse reaches. Here one kernel runs over
// the step's manifold list right before the solver, on the same velocities its constraint data is built from, and
// appends the events to a ring with one atomic per warp; each record carries its manifold index and side, and the
// host puts the events in manifold order (side a before side b) before dispatching them, so the order does not
// depend on scheduling. A ring too small for the step sets STATUS_EVENT_OVERFLOW and counts every event, and the
// host grows it and steps again.
#include "ag2d_kernels.cuh"
#include "ag2d_solver.cuh"

namespace ag2d {

__global__ void k_collision_events(DeviceWorld w, const ColliderEvent* __restrict__ cev,
                                   const Manifold* __restrict__ man, const uint32_t* __restrict__ nMan,
                                   uint32_t manCap, EventRecord* __restrict__ ring, uint32_t ringCap,
                                   StepCounters* counters)
{
    const uint32_t n = min(*nMan, manCap);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t warpsTotal = (gridDim.x * blockDim.x) >> 5;
    // Whole warps step through the list together (their ballots need every lane).
    for (uint32_t base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) << 5; base < n; base += warpsTotal << 5) {
        const uint32_t i = base + lane;
        bool fireA = false, fireB = false;
        Manifold m;
        float impact = 0.0f;
        uint32_t bA = 0, bB = 0;
        ColliderEvent eA{0u, 0.0f}, eB{0u, 0.0f};
        if (i < n) {
            const uint2 ab = *reinterpret_cast<const uint2*>(man + i);
            eA = cev[ab.x];
            eB = cev[ab.y];
            if (eA.callback != 0u || eB.callback != 0u) {
                m = man[i];
                bA = w.cbody[m.a];
                bB = w.cbody[m.b];
                impact = impact_impulse(m, w.bvel[bA], w.bvel[bB], w.bpos[bA], w.bpos[bB]);
                if (impact > 0.0f) {
                    fireA = eA.callback != 0u && impact >= eA.threshold;
                    fireB = eB.callback != 0u && impact >= eB.threshold;
                }
            }
        }
        const uint32_t ballotA = __ballot_sync(0xffffffffu, fireA);
        const uint32_t ballotB = __ballot_sync(0xffffffffu, fireB);
        const uint32_t total = __popc(ballotA) + __popc(ballotB);
        if (total == 0u) continue;
        uint32_t slot0 = 0u;
        if (lane == 0) {
            slot0 = atomicAdd(&counters->events, total);
            if (slot0 + total > ringCap) atomicOr(&counters->status, STATUS_EVENT_OVERFLOW);
        }
        slot0 = __shfl_sync(0xffffffffu, slot0, 0);
        if (!fireA && !fireB) continue;
        uint32_t slot = slot0 + __popc(ballotA & lt) + __popc(ballotB & lt);
        // Event point: the average of the two contact points, or the only one (BodyCollisionSolver.cpp:363-365).
        const float px = m.count > 1 ? (m.px0 + m.px1) * 0.5f : m.px0;
        const float py = m.count > 1 ? (m.py0 + m.py1) * 0.5f : m.py0;
        if (fireA) {
            if (slot < ringCap) {
                EventRecord r;
                r.manifold = i; r.side = 0u; r.self = m.a; r.other = m.b; r.selfBody = bA; r.otherBody = bB;
                r.callback = eA.callback; r.impulse = impact; r.px = px; r.py = py; r.nx = m.nx; r.ny = m.ny;
                ring[slot] = r;
            }
            slot++;
        }
        if (fireB && slot < ringCap) {
            EventRecord r;
            r.manifold = i; r.side = 1u; r.self = m.b; r.other = m.a; r.selfBody = bB; r.otherBody = bA;
            r.callback = eB.callback; r.impulse = impact; r.px = px; r.py = py; r.nx = -m.nx; r.ny = -m.ny;
            ring[slot] = r;
        }
    }
}

}  // namespace ag2d
