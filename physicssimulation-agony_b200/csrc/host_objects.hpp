// Host-side object bookkeeping: body/collider/shape creation with the reference's geometry and dense ordering.
//
// Creation is host work in the reference too (ObjectManager, PhysicsGeometry). What matters for parity is
// reproduced exactly: mass/inertia/centre-of-mass arithmetic (SimulationImpl/PhysicsGeometry.cpp:116-187),
// polygon outline cleaning for convex input (:275-347) and recentring (ObjectManager.cpp:286-349, 535-562), the
// bound radius (ObjectManager.cpp:24-43, 1103-1108), and the dense order that group moves produce
// (moveBodyToGroup, ObjectManager.cpp:1232-1267): a new static body takes the first slot after the static group
// and pushes the first body of each later group to that group's end. Paths are relative to
// PhysicsSimulation-Agony/PS_AGONY2D/.
#pragma once

#include <cmath>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace ag2d {

struct HBody {
    float comX = 0, comY = 0, vx = 0, vy = 0, rot = 0, w = 0;
    float mass = 0, invMass = 0, inertia = 0, invInertia = 0;
    float lcomX = 0, lcomY = 0;
    float cos = 1, sin = 0;
    float boundRadius = 0;
    float wrapCount = 0, sleepTimer = 0;
    uint32_t sleepIsland = 0xFFFFFFFFu;
    uint32_t handleSlot = 0;
    std::vector<uint32_t> colliders;
};

struct HCollider {
    uint32_t body = 0;
    float locX = 0, locY = 0, comOffX = 0, comOffY = 0, localRot = 0;
    uint32_t material = 0;
    uint32_t type = 0, shape = 0;
    float minExtent = 0, maxExtent = 0;
    // Collision-event opt-in (ColliderSoA callbackId / eventThreshold, SoA/ColliderSoA.cpp:47-48): no callback and
    // the never-firing threshold (NO_COLLISION_EVENT_THRESHOLD, Types/CollisionEvent.h:15) at creation. It moves
    // with the collider when the dense order changes.
    uint32_t callback = 0;
    float eventThreshold = 3.40282347e38f;
};

struct HPolygon {
    std::vector<float> verts;     // xy pairs, collider-local, centred on the piece centroid
    std::vector<float> normals;   // xy pairs, outward unit edge normals (0 for degenerate edges)
};

// Group ranges: [starts[g], starts[g + 1]) for static (0), sleeping (1), dynamic (2); starts[3] = live count.
struct Groups {
    uint32_t starts[4] = {0, 0, 0, 0};
    uint32_t groupOf(uint32_t i) const
    {
        for (uint32_t g = 0; g < 3; g++) if (i < starts[g + 1]) return g;
        return 3;
    }
};

// Constraints between bodies (SimulationImpl/ConstraintSystems/*, SoA/Constraints/*): springs, revolute, prismatic
// and slider joints, motors. A system keeps its constraints in the reference's dense order, grouped [Inactive][Sleeping][Active]
// (ConstraintGroup, ConstraintSystemBase.h:22-24; Inactive: every body static), moved between groups by the same
// boundary swaps (ObjectManager::moveConstraintToGroup, ObjectManager.cpp:1172-1205), with a handle table whose
// freed slots are reused last-in first-out with the generation raised (HandleTable.h:30-90).
enum JointKind : uint32_t {
    JOINT_SPRING = 0, JOINT_REVOLUTE = 1, JOINT_PRISMATIC = 2, JOINT_SLIDER = 3, JOINT_MOTOR = 4, JOINT_KINDS = 5
};
enum JointGroup : uint32_t { JGROUP_INACTIVE = 0, JGROUP_SLEEPING = 1, JGROUP_ACTIVE = 2, JGROUP_UNUSED = 3 };
constexpr uint32_t NO_BODY = 0xFFFFFFFFu;

struct HJoint {
    uint32_t bodyA = 0, bodyB = NO_BODY;   // dense body indices (motors: bodyA only)
    float anchorAx = 0, anchorAy = 0, anchorBx = 0, anchorBy = 0;   // body-local anchors
    float restLength = 0, stiffness = 0, damping = 0;               // spring (revolute: stiffness, damping)
    float targetSpeed = 0, maxTorque = 0, impulse = 0;              // motor; impulse: accumulated (warm start)
    float axisX = 1, axisY = 0;                                       // prismatic / slider: body A's local axis
    float referenceAngle = 0;                                         // prismatic: locked relative angle
    float lowerLimit = 0, upperLimit = 0;                             // prismatic / slider: axis limits
    bool enableLimit = false;
    uint32_t handleSlot = 0;
};

struct JointSystem {
    std::vector<HJoint> joints;
    uint32_t starts[4] = {0, 0, 0, 0};   // first index of each group; starts[3]: end of the live constraints
    uint32_t iterations = 6;             // IConstraintSystem::iterations (ConstraintSystemBase.h:34)
    std::vector<uint32_t> slotIndex, slotGeneration;
    uint32_t freeHead = NO_BODY;

    uint32_t groupOf(uint32_t i) const
    {
        for (uint32_t g = 0; g < 3; g++) if (i >= starts[g] && i < starts[g + 1]) return g;
        return JGROUP_UNUSED;
    }
    uint32_t indexOf(uint64_t handle) const
    {
        const uint32_t slot = uint32_t(handle & 0xFFFFFFFFu), gen = uint32_t(handle >> 32);
        if (slot >= slotIndex.size() || slotGeneration[slot] != gen || slotIndex[slot] == NO_BODY) return NO_BODY;
        return slotIndex[slot];
    }
    uint64_t handleOf(uint32_t i) const
    {
        const uint32_t slot = joints[i].handleSlot;
        return (uint64_t(slotGeneration[slot]) << 32) | slot;
    }
    // Appends and moves the constraint to 'group' (createConstraint + refreshConstraintGroup,
    // ObjectManager.cpp:430-475, 1207-1220). Returns its dense index.
    uint32_t create(const HJoint& j, uint32_t group);
    // Moves to the unused group and pops (destroyConstraintInternal, ObjectManager.cpp:502-520).
    void destroy(uint32_t index);
    uint32_t moveToGroup(uint32_t index, uint32_t group);
    void swap(uint32_t a, uint32_t b);
};

class HostObjects {
public:
    JointSystem jointSystems[JOINT_KINDS];
    std::vector<HBody> bodies;
    std::vector<HCollider> colliders;
    std::vector<float> circleRadius;
    std::vector<float> boxHalfW, boxHalfH;   // boxes' half extents; capsules share the table: half length, radius
    std::vector<HPolygon> polygons;
    std::vector<float> materials;   // 3 per material
    Groups bodyGroups, colGroups;
    // Handle table: slot -> dense index (generation kept beside it).
    std::vector<uint32_t> slotIndex, slotGeneration;

    HostObjects() { materials = {1.0f, 0.0f, 0.0f}; }   // MaterialManager: material 0 = default

    uint32_t addMaterial(float e, float sf, float df)
    {
        // MaterialManager::sanitize (SimulationImpl/MaterialManager.h:29-35).
        e = std::fmin(std::fmax(e, 0.0f), 1.0f);
        sf = std::fmax(sf, 0.0f);
        df = std::fmax(df, 0.0f);
        materials.push_back(e); materials.push_back(sf); materials.push_back(df);
        return uint32_t(materials.size() / 3 - 1);
    }
    uint32_t materialCount() const { return uint32_t(materials.size() / 3); }

    // Returns the handle ((generation << 32) | slot) or sets err.
    bool addCircle(const float* desc /* x,y,rot,vx,vy,w,mass */, uint32_t material, float radius, uint64_t& handle,
                   std::string& err);
    bool addBox(const float* desc, uint32_t material, float width, float height, uint64_t& handle, std::string& err);
    bool addPolygon(const float* desc, uint32_t material, const float* xy, uint32_t n, uint64_t& handle,
                    std::string& err);
    bool addCapsule(const float* desc, uint32_t material, float length, float radius, uint64_t& handle,
                    std::string& err);
    // ObjectManager::createBody (ObjectManager.cpp:71-88): a body with explicit mass, inertia and local centre of
    // mass and no collider yet.
    bool addBody(const float* desc, float inertia, float comX, float comY, uint64_t& handle, std::string& err);
    // ObjectManager::create{Circle,Box,Polygon,Capsule}Collider (ObjectManager.cpp:90-231): a collider on an
    // existing body, at a local offset and rotation; p holds radius / (width, height) / (length, radius). Polygons
    // are convex outlines (xy, n), recentred on their centroid with the shift added to the offset. Returns the
    // collider's dense index.
    bool addCollider(uint32_t body, uint32_t type, float locX, float locY, float localRot, uint32_t material,
                     const float* p, const float* xy, uint32_t n, uint32_t& collider, std::string& err);

    // colliderArea (ObjectManager.cpp:593-612) with PhysicsGeometry's areas (PhysicsGeometry.cpp:115-144).
    float colliderArea(uint32_t c) const;
    // A collider's inertia about its own origin for mass m (PhysicsGeometry::calculate*Inertia at the origin, as
    // ObjectManager::recomputeBodyInertia takes them, ObjectManager.cpp:917-970).
    float colliderOwnInertia(uint32_t c, float m) const;
    // refreshBoundRadius (ObjectManager.cpp:37-43): the farthest reach of the body's colliders from its centre.
    float boundRadiusOf(uint32_t b) const;

    uint32_t indexOf(uint64_t handle) const
    {
        const uint32_t slot = uint32_t(handle & 0xFFFFFFFFu), gen = uint32_t(handle >> 32);
        if (slot >= slotIndex.size() || slotGeneration[slot] != gen) return 0xFFFFFFFFu;
        return slotIndex[slot];
    }

private:
    uint32_t appendBody(float px, float py, float vx, float vy, float rot, float w, float mass, float invMass,
                        float inertia, float invInertia, float lcomX, float lcomY);
    uint32_t appendCollider(uint32_t body, float locX, float locY, float localRot, uint32_t material, uint32_t type,
                            uint32_t shape, float minExt, float maxExt);
    uint32_t appendPolygonPiece(uint32_t body, float offX, float offY, float localRot, uint32_t material,
                                std::vector<float> outline);
    void swapBodies(uint32_t a, uint32_t b);
    void swapColliders(uint32_t a, uint32_t b);
    uint32_t moveBodyDown(uint32_t index, uint32_t target);
    uint32_t moveColliderDown(uint32_t index, uint32_t target);
};

// PhysicsGeometry::calculatePolygonInertia (PhysicsGeometry.cpp:130-187) without a requested pivot.
// Returns false for a degenerate (or clockwise) outline.
bool polygon_inertia(float mass, const std::vector<float>& xy, float& inertia, float& cx, float& cy);

// PhysicsGeometry::preparePolygonOutline (PhysicsGeometry.cpp:175-212): duplicates and straight vertices dropped,
// made counter-clockwise; false with a reason for a degenerate or non-simple outline. Concave outlines pass.
bool prepare_outline_any(const float* xy, uint32_t n, std::vector<float>& out, std::string& err);

// prepare_outline_any for a convex outline of at most 16 vertices (ObjectManager::queueColliderPolygon's checks,
// ObjectManager.cpp:622-636); false with a reason otherwise.
bool prepare_outline(const float* xy, uint32_t n, std::vector<float>& out, std::string& err);

// isConvexPolygon and isSimplePolygon (PolygonDecomposition.cpp:618-671) on xy pairs.
bool outline_is_convex(const std::vector<float>& xy);
bool outline_is_simple(const std::vector<float>& xy);

// PhysicsGeometry::decomposeConcave with the Bayazit method (ear clipping when it finds no diagonal), then
// limitConvexPieceVertexCount with the fan split (PolygonDecomposition.cpp:704-831): convex pieces (xy pairs, the
// prepared outline's vertices) of at most maxVertices vertices each.
std::vector<std::vector<float>> decompose_outline(const std::vector<float>& xy, size_t maxVertices);

// PolygonGeometry::computeNormals (SoA/Shapes/PolygonSoA.cpp:14-30): outward unit edge normals as xy pairs.
std::vector<float> polygon_normals(const std::vector<float>& v);

}  // namespace ag2d
