// C++ facade over the C ABI of libag2d.so with the names and call shapes of PS_AGONY2D's public API, so scene code
// written against the reference's Simulation / ObjectAPI compiles against this library with a namespace change.
//
//   reference                                   here
//   PS_AGONY2D::Simulation (Simulation.h:36)    ag2d::Simulation      update, createMaterial, objects,
//                                                                     getBodyCollisionData, getSimulationSettings
//   PS_AGONY2D::ObjectAPI (ObjectAPI.h:14)      ag2d::ObjectAPI       createCircle/Box/Polygon (+ H variants),
//                                                                     getBodyIndex, getBodies
//   ConstraintAPI (ConstraintAPI.h:13)          ag2d::ConstraintAPI   create/destroy springs, revolute, prismatic
//                                                                     and slider joints, motors; their setters
//   Simulation collision callbacks              createCollisionCallback, destroyCollisionCallback,
//   (Simulation.h:169-179)                      setColliderCollisionCallback, getCollisionEvents
//   SimulationSettings (Simulation.h:50-76)     ag2d::SimulationSettings
//   FixedClock (SimulationImpl/FixedClock.h)    the same accumulator semantics inside Simulation::update
//   Body/Circle/Box/PolygonCreateParams         same fields (SimulationImpl/ObjectCreateParams.h:14-95)
//
// Creation failures return std::nullopt like the reference (ObjectManager.cpp:92-97); device and capacity errors
// throw std::runtime_error carrying ag2d_last_error_string(). Header-only; link with -lag2d.
#pragma once

#include "ag2d.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ag2d {

using Real = float;
using ObjectDenseIndex = uint32_t;
using MaterialIndex = uint32_t;

struct Vec2 {
    Real x = 0, y = 0;
};

// A body handle as the C ABI returns it (slot and generation packed in 64 bits).
struct Handle {
    uint64_t value = 0;
};

struct Material {
    Real elasticity = 1;
    Real staticFriction = 0;
    Real dynamicFriction = 0;
};

struct BodyCreateParams {
    Vec2 position{};
    Vec2 velocity{};
    Real rotation = 0;
    Real angularVelocity = 0;
    Real mass = 0;          // 0: a static body
    Real inertia = 0;       // create<Shape>: must be 0 (inertia from the shape); createBody: the body's inertia
    std::optional<Vec2> centerOfMass = std::nullopt;   // createBody only: local centre of mass (default origin)
    MaterialIndex materialIndex = 0;
};
// Collider params (SimulationImpl/ObjectCreateParams.h:26-69): a shape attached to an existing body at a local offset
// and rotation. Concave polygons become one collider per convex piece, as in the reference; capsules take the
// length / radius form.
struct ColliderCreateParams {
    Handle bodyHandle;
    Vec2 localOffset{};
    Real localRotation = 0;
    MaterialIndex materialIndex = 0;
};
struct CircleColliderCreateParams : ColliderCreateParams {
    Real radius = 0;
};
struct BoxColliderCreateParams : ColliderCreateParams {
    Vec2 size{};
};
struct PolygonColliderCreateParams : ColliderCreateParams {
    std::span<const Vec2> localVertices;
};
struct PolygonColliderCreateResult {
    ObjectDenseIndex firstColliderIndex{0};
    size_t colliderCount{0};
};
struct CapsuleColliderCreateParams : ColliderCreateParams {
    Real length = 0;
    Real radius = 0;
};
struct CircleCreateParams {
    BodyCreateParams base;
    Real radius = 0;
};
struct BoxCreateParams {
    BodyCreateParams base;
    Vec2 size{};
};
struct PolygonCreateParams {
    BodyCreateParams base;
    std::span<Vec2> localVertices;
};
// CapsuleCreateParams (SimulationImpl/ObjectCreateParams.h:98-105) without the endpoint form: a core of 'length'
// along the body's x axis, swept by 'radius'.
struct CapsuleCreateParams {
    BodyCreateParams base;
    Real length = 0;
    Real radius = 0;
};

struct FixedClockSettings {
    Real updateInterval = Real(1) / Real(300);
    Real maxDeltaTimePerUpdateCall = Real(1) / Real(20);
    Real timeScale = Real(1);
};
struct IntegratorSettings {
    Vec2 gravity{0, Real(-9.81)};
    Real angularVelocityDamping = 1;   // 1: off
};
// Collision events (Types/CollisionEvent.h:10-31). Colliders are named by dense index, which is stable in this
// library (the reference names them by collider handle); bodies by handle.
using CollisionCallbackIndex = uint16_t;
inline constexpr Real NO_COLLISION_EVENT_THRESHOLD = std::numeric_limits<Real>::max();
struct CollisionEvent {
    ObjectDenseIndex self = 0, other = 0;
    Handle selfBody, otherBody;
    Vec2 point;      // average of the manifold's contact points
    Vec2 normal;     // from self towards other
    Real impulse = 0;   // impact impulse: max over the contacts of approach speed x normal effective mass, pre-solve
    CollisionCallbackIndex callbackId = 0;
};
// Constraint creation parameters (SimulationImpl/ConstraintSystems/*ConstraintSystem.h: CreateParams), under the
// reference's class names.
struct SpringConstraintSystem {
    struct CreateParams {
        Handle bodyHandleA, bodyHandleB;
        Vec2 localAnchorA, localAnchorB;
        Real restLength = 0, stiffness = 0, damping = 0;
    };
};
struct RevoluteJointConstraintSystem {
    struct CreateParams {
        Handle bodyHandleA, bodyHandleB;
        Vec2 localAnchorA, localAnchorB;
        Real stiffness = 0, damping = 0;
    };
};
struct PrismaticJointConstraintSystem {
    struct CreateParams {
        Handle bodyHandleA, bodyHandleB;
        Vec2 localAnchorA, localAnchorB;
        Vec2 localAxisA{1, 0};
        Real stiffness = 0, damping = 0;
        Real lowerLimit = 0, upperLimit = 0;
        bool enableLimit = false;
    };
};
struct SliderJointConstraintSystem {
    using CreateParams = PrismaticJointConstraintSystem::CreateParams;
};
struct MotorConstraintSystem {
    struct CreateParams {
        Handle bodyHandle;
        Real targetSpeed = 0, maxTorque = 0;
    };
};

class Simulation;
using CollisionCallback = void (*)(const CollisionEvent& event, Simulation& simulation, void* userData);

struct SimulationSettings {
    FixedClockSettings clockSettings;
    uint32_t collisionVelocitySolvingIterations = 6;
    uint32_t collisionPositionSolvingIterations = 3;
    IntegratorSettings integratorSettings;
    bool continuousCollisionEnabled = true;
    Real sleepSpeedThreshold = Real(0.1);
    Real sleepTimeThreshold = Real(0.5);
    bool collisionEventsEnabled = true;        // also requires at least one collision callback
    int device = 0;                            // CUDA device ordinal
};

// Host copy of the body arrays in dense order (the reference's BodySoAViewer fields used by scene code).
struct BodyView {
    std::vector<Real> comX, comY, rotation, velocityX, velocityY, angularVelocity;
    uint32_t getCount() const { return uint32_t(comX.size()); }
};

namespace detail {
inline void check(int32_t code)
{
    if (code != AG2D_OK) throw std::runtime_error(std::string("ag2d: ") + ag2d_last_error_string());
}
inline ag2d_body_desc desc(const BodyCreateParams& b)
{
    ag2d_body_desc d{};
    d.x = b.position.x; d.y = b.position.y; d.rotation = b.rotation;
    d.vx = b.velocity.x; d.vy = b.velocity.y; d.angular_velocity = b.angularVelocity;
    d.mass = b.mass; d.material = b.materialIndex;
    return d;
}
inline std::vector<float> read_floats(ag2d_world* w, int32_t field)
{
    uint64_t bytes = 0;
    check(ag2d_world_read(w, field, nullptr, 0, &bytes));
    std::vector<float> v(bytes / sizeof(float));
    check(ag2d_world_read(w, field, v.data(), bytes, &bytes));
    return v;
}
}  // namespace detail

class ObjectAPI {
public:
    explicit ObjectAPI(ag2d_world* w) : world(w) {}
    ObjectAPI(const ObjectAPI&) = delete;
    ObjectAPI& operator=(const ObjectAPI&) = delete;

    std::optional<ObjectDenseIndex> createCircle(const CircleCreateParams& p) { return index(createCircleH(p)); }
    std::optional<ObjectDenseIndex> createBox(const BoxCreateParams& p) { return index(createBoxH(p)); }
    std::optional<ObjectDenseIndex> createPolygon(const PolygonCreateParams& p) { return index(createPolygonH(p)); }
    std::optional<ObjectDenseIndex> createCapsule(const CapsuleCreateParams& p) { return index(createCapsuleH(p)); }

    std::optional<Handle> createCircleH(const CircleCreateParams& p)
    {
        if (p.base.inertia != 0) return std::nullopt;
        const ag2d_body_desc d = detail::desc(p.base);
        uint64_t h = 0;
        const int32_t code = ag2d_world_add_circle(world, &d, p.radius, &h);
        return created(code, h);
    }
    std::optional<Handle> createBoxH(const BoxCreateParams& p)
    {
        if (p.base.inertia != 0) return std::nullopt;
        const ag2d_body_desc d = detail::desc(p.base);
        uint64_t h = 0;
        const int32_t code = ag2d_world_add_box(world, &d, p.size.x, p.size.y, &h);
        return created(code, h);
    }
    std::optional<Handle> createPolygonH(const PolygonCreateParams& p)
    {
        if (p.base.inertia != 0) return std::nullopt;
        const ag2d_body_desc d = detail::desc(p.base);
        std::vector<float> xy;
        xy.reserve(p.localVertices.size() * 2);
        for (const Vec2& v : p.localVertices) { xy.push_back(v.x); xy.push_back(v.y); }
        uint64_t h = 0;
        const int32_t code = ag2d_world_add_polygon(world, &d, xy.data(), uint32_t(p.localVertices.size()), &h);
        return created(code, h);
    }

    std::optional<Handle> createCapsuleH(const CapsuleCreateParams& p)
    {
        if (p.base.inertia != 0) return std::nullopt;
        const ag2d_body_desc d = detail::desc(p.base);
        uint64_t h = 0;
        const int32_t code = ag2d_world_add_capsule(world, &d, p.length, p.radius, &h);
        return created(code, h);
    }

    // ObjectAPI::createBody / createBodyH (ObjectAPI.h:28, 61): a body with explicit mass, inertia and centre of
    // mass and no collider; colliders are attached with create*Collider (ObjectAPI.h:29-32), which return the new
    // collider's dense index.
    std::optional<ObjectDenseIndex> createBody(const BodyCreateParams& p) { return index(createBodyH(p)); }
    std::optional<Handle> createBodyH(const BodyCreateParams& p)
    {
        const ag2d_body_desc d = detail::desc(p);
        const Vec2 com = p.centerOfMass.value_or(Vec2{});
        uint64_t h = 0;
        const int32_t code = ag2d_world_create_body(world, &d, p.inertia, com.x, com.y, &h);
        return created(code, h);
    }
    std::optional<ObjectDenseIndex> createCircleCollider(const CircleColliderCreateParams& p)
    {
        const float params[2] = {p.radius, 0};
        return collider(p, 0, params, nullptr, 0);
    }
    std::optional<ObjectDenseIndex> createBoxCollider(const BoxColliderCreateParams& p)
    {
        const float params[2] = {p.size.x, p.size.y};
        return collider(p, 1, params, nullptr, 0);
    }
    // The first piece's index and the number of convex pieces (colliders) the outline became
    // (PolygonColliderCreateResult, ObjectCreateParams.h:71-75); the pieces follow the first in the body's colliders.
    std::optional<PolygonColliderCreateResult> createPolygonCollider(const PolygonColliderCreateParams& p)
    {
        std::vector<float> xy;
        xy.reserve(p.localVertices.size() * 2);
        for (const Vec2& v : p.localVertices) { xy.push_back(v.x); xy.push_back(v.y); }
        const uint32_t n = uint32_t(p.localVertices.size());
        const std::optional<ObjectDenseIndex> first = collider(p, 2, nullptr, xy.data(), n);
        if (!first) return std::nullopt;
        uint32_t pieces = 0;   // the count alone: no output arrays (AG2D_ERR_CAPACITY with the count written)
        ag2d_decompose_polygon(xy.data(), n, nullptr, 0, nullptr, 0, &pieces);
        return PolygonColliderCreateResult{*first, size_t(pieces)};
    }
    std::optional<ObjectDenseIndex> createCapsuleCollider(const CapsuleColliderCreateParams& p)
    {
        const float params[2] = {p.length, p.radius};
        return collider(p, 3, params, nullptr, 0);
    }

    // Deferred body commands (ObjectAPI.h:72-81): applied at the start of the next update's first step; stale
    // handles are dropped then. A destroyed body keeps its dense index with state AG2D_BODY_DESTROYED.
    void destroyBody(Handle h) { detail::check(ag2d_world_destroy_body(world, h.value)); }
    void setBodyPosition(Handle h, Vec2 p) { detail::check(ag2d_world_set_body_position(world, h.value, p.x, p.y)); }
    void setBodyRotation(Handle h, Real r) { detail::check(ag2d_world_set_body_rotation(world, h.value, r)); }
    void setBodyVelocity(Handle h, Vec2 v) { detail::check(ag2d_world_set_body_velocity(world, h.value, v.x, v.y)); }
    void setBodyAngularVelocity(Handle h, Real w)
    {
        detail::check(ag2d_world_set_body_angular_velocity(world, h.value, w));
    }
    void setBodyMass(Handle h, Real m) { detail::check(ag2d_world_set_body_mass(world, h.value, m)); }
    void setBodyInertia(Handle h, Real i) { detail::check(ag2d_world_set_body_inertia(world, h.value, i)); }
    void setBodyLocalCenterOfMass(Handle h, Vec2 c)
    {
        detail::check(ag2d_world_set_body_local_center_of_mass(world, h.value, c.x, c.y));
    }
    void recomputeBodyInertia(Handle h) { detail::check(ag2d_world_recompute_body_inertia(world, h.value)); }
    void setBodyMassFromDensity(Handle h, Real d)
    {
        detail::check(ag2d_world_set_body_mass_from_density(world, h.value, d));
    }
    // Collider setters (ObjectAPI.h:86-91) by dense collider index (the reference takes the collider's handle;
    // collider indices are stable here). Deferred to the next step like the body commands.
    void setColliderLocalOffset(ObjectDenseIndex c, Vec2 o) { collider(c, AG2D_COMMAND_COLLIDER_OFFSET, o.x, o.y); }
    void setColliderLocalRotation(ObjectDenseIndex c, Real r) { collider(c, AG2D_COMMAND_COLLIDER_ROTATION, r, 0); }
    void setColliderMaterial(ObjectDenseIndex c, MaterialIndex m)
    {
        collider(c, AG2D_COMMAND_COLLIDER_MATERIAL, Real(m), 0);
    }
    void setCircleRadius(ObjectDenseIndex c, Real r) { collider(c, AG2D_COMMAND_CIRCLE_RADIUS, r, 0); }
    void setBoxSize(ObjectDenseIndex c, Vec2 size) { collider(c, AG2D_COMMAND_BOX_SIZE, size.x, size.y); }
    void setCapsuleShape(ObjectDenseIndex c, Real length, Real radius)
    {
        collider(c, AG2D_COMMAND_CAPSULE_SHAPE, length, radius);
    }
    // ObjectAPI::setPolygonShape (ObjectAPI.h:93): false, with nothing queued, for an outline the reference refuses
    // (fewer than 3 vertices, degenerate, concave, more than 16 vertices).
    bool setPolygonShape(ObjectDenseIndex c, std::span<const Vec2> localVertices)
    {
        std::vector<float> xy;
        xy.reserve(localVertices.size() * 2);
        for (const Vec2& v : localVertices) { xy.push_back(v.x); xy.push_back(v.y); }
        const int32_t code = ag2d_world_set_polygon_shape(world, c, xy.data(), uint32_t(localVertices.size()));
        if (code == AG2D_ERR_INVALID_ARG) return false;
        detail::check(code);
        return true;
    }

    // Dense index of a handle; UINT32_MAX when the handle is stale (ObjectAPI::getBodyIndex, ObjectAPI.h:53).
    ObjectDenseIndex getBodyIndex(Handle h) const noexcept { return ag2d_world_body_index(world, h.value); }

    BodyView getBodies() const
    {
        BodyView v;
        v.comX = detail::read_floats(world, AG2D_BODY_COM_X);
        v.comY = detail::read_floats(world, AG2D_BODY_COM_Y);
        v.rotation = detail::read_floats(world, AG2D_BODY_ROTATION);
        v.velocityX = detail::read_floats(world, AG2D_BODY_VEL_X);
        v.velocityY = detail::read_floats(world, AG2D_BODY_VEL_Y);
        v.angularVelocity = detail::read_floats(world, AG2D_BODY_ANGULAR_VELOCITY);
        return v;
    }

private:
    void collider(ObjectDenseIndex c, int32_t command, Real a, Real b)
    {
        detail::check(ag2d_world_set_collider(world, c, command, a, b));
    }
    // Invalid shapes (the reference's nullopt cases) return nullopt; anything else is an error.
    // 'code' is the creating call's result, evaluated before 'h' is read (the call writes h).
    static std::optional<Handle> created(int32_t code, uint64_t h)
    {
        if (code == AG2D_ERR_INVALID_ARG || code == AG2D_ERR_UNSUPPORTED) return std::nullopt;
        detail::check(code);
        return Handle{h};
    }
    std::optional<ObjectDenseIndex> index(std::optional<Handle> h) const
    {
        if (!h) return std::nullopt;
        return getBodyIndex(*h);
    }
    // Failures the reference reports with an empty optional (stale body handle, degenerate or unsupported outline)
    // come back the same way; others throw.
    std::optional<ObjectDenseIndex> collider(const ColliderCreateParams& p, int32_t shape, const float* params,
                                             const float* xy, uint32_t n)
    {
        uint32_t c = 0;
        const int32_t code = ag2d_world_add_collider(world, p.bodyHandle.value, shape, p.localOffset.x,
                                                     p.localOffset.y, p.localRotation, p.materialIndex, params, xy,
                                                     n, &c);
        if (code == AG2D_ERR_INVALID_ARG || code == AG2D_ERR_UNSUPPORTED) return std::nullopt;
        detail::check(code);
        return c;
    }
    ag2d_world* world;
};

struct AABB {
    Real minX = 0, minY = 0, maxX = 0, maxY = 0;
};

// Query shapes of the broad phase (CollisionDetection/Broad/QueryShapes.h:8-86) and its tree selection flags
// (BvhTree.h:26-33).
namespace BroadPhaseInternal {
enum class BvhTreeTypeFlag : uint8_t { None = 0, Dynamic = 1, Static = 2, Sleeping = 4, All = 7 };
constexpr BvhTreeTypeFlag operator|(BvhTreeTypeFlag a, BvhTreeTypeFlag b) noexcept
{
    return BvhTreeTypeFlag(uint8_t(a) | uint8_t(b));
}
struct AABBQuery {
    AABB aabb;
    explicit AABBQuery(const AABB& a) noexcept : aabb(a) {}
};
struct CircleQuery {
    Vec2 pos;
    Real radius;
    CircleQuery(Vec2 p, Real r) noexcept : pos(p), radius(r) {}
};
}  // namespace BroadPhaseInternal

// The broad phase's spatial queries (BroadPhaseCollisionDetector::queryCollidersInShape,
// BroadPhaseCollisionDetector.h:164-203). Indices are this library's collider indices; the found set is the
// reference's, appended in ascending index order.
class BroadPhaseCollisionDetector {
public:
    explicit BroadPhaseCollisionDetector(ag2d_world* w) : world(w) {}
    void queryCollidersInShape(const BroadPhaseInternal::AABBQuery& q, BroadPhaseInternal::BvhTreeTypeFlag flags,
                               std::vector<ObjectDenseIndex>& out) const
    {
        const float p[4] = {q.aabb.minX, q.aabb.minY, q.aabb.maxX, q.aabb.maxY};
        run(AG2D_QUERY_AABB, p, flags, out);
    }
    void queryCollidersInShape(const BroadPhaseInternal::CircleQuery& q, BroadPhaseInternal::BvhTreeTypeFlag flags,
                               std::vector<ObjectDenseIndex>& out) const
    {
        const float p[4] = {q.pos.x, q.pos.y, q.radius, 0.0f};
        run(AG2D_QUERY_CIRCLE, p, flags, out);
    }

private:
    void run(int32_t shape, const float* p, BroadPhaseInternal::BvhTreeTypeFlag flags,
             std::vector<ObjectDenseIndex>& out) const
    {
        uint32_t n = 0;
        detail::check(ag2d_world_query_shape(world, shape, p, uint32_t(flags), nullptr, 0, &n));
        const size_t base = out.size();
        out.resize(base + n);
        if (n) detail::check(ag2d_world_query_shape(world, shape, p, uint32_t(flags), out.data() + base, n, &n));
    }
    ag2d_world* world;
};

// The narrow phase's circle test (NarrowPhaseCollisionDetector::findCollisionsInCircle,
// NarrowPhaseCollisionDetector.cpp:153-270): for each collider of 'collidersToCheck' that the circle touches, its
// index and the signed distance from the circle's centre, in the order given.
class NarrowPhaseCollisionDetector {
public:
    explicit NarrowPhaseCollisionDetector(ag2d_world* w) : world(w) {}
    void findCollisionsInCircle(std::span<const ObjectDenseIndex> collidersToCheck, Vec2 pos, Real radius,
                                std::vector<std::pair<ObjectDenseIndex, Real>>& outColliding) const
    {
        // The device answers over the colliders whose broad-phase AABBs (those of the last step) pass the circle
        // query, filtered to the colliders given. Between steps the AABBs are current, so that set holds every
        // collider the circle touches; a collider moved since the last step by a command is only seen from the next
        // step on (the reference tests every given collider at its current pose).
        uint32_t n = 0;
        detail::check(ag2d_world_query_circle_contacts(world, pos.x, pos.y, radius, AG2D_TREE_ALL, nullptr, nullptr, 0,
                                                        &n));
        std::vector<uint32_t> idx(n);
        std::vector<float> dist(n);
        if (n) detail::check(ag2d_world_query_circle_contacts(world, pos.x, pos.y, radius, AG2D_TREE_ALL, idx.data(),
                                                               dist.data(), n, &n));
        for (ObjectDenseIndex c : collidersToCheck) {
            const auto it = std::lower_bound(idx.begin(), idx.end(), c);   // ascending indices
            if (it != idx.end() && *it == c) outColliding.emplace_back(c, Real(dist[size_t(it - idx.begin())]));
        }
    }

private:
    ag2d_world* world;
};

// ConstraintAPI (SimulationAPIs/ConstraintAPI.h:13-105): creation returns a handle (nullopt for a stale body
// handle); destroys and edits are deferred to the next step, as in the reference.
class ConstraintAPI {
public:
    explicit ConstraintAPI(ag2d_world* w) : world(w) {}
    ConstraintAPI(const ConstraintAPI&) = delete;
    ConstraintAPI& operator=(const ConstraintAPI&) = delete;

    std::optional<Handle> createSpring(const SpringConstraintSystem::CreateParams& p)
    {
        ag2d_joint_desc d = pair(AG2D_JOINT_SPRING, p.bodyHandleA, p.bodyHandleB, p.localAnchorA, p.localAnchorB);
        d.rest_length = p.restLength; d.stiffness = p.stiffness; d.damping = p.damping;
        return create(d);
    }
    std::optional<Handle> createRevoluteJoint(const RevoluteJointConstraintSystem::CreateParams& p)
    {
        ag2d_joint_desc d = pair(AG2D_JOINT_REVOLUTE, p.bodyHandleA, p.bodyHandleB, p.localAnchorA, p.localAnchorB);
        d.stiffness = p.stiffness; d.damping = p.damping;
        return create(d);
    }
    std::optional<Handle> createPrismaticJoint(const PrismaticJointConstraintSystem::CreateParams& p)
    {
        return create(axisJoint(AG2D_JOINT_PRISMATIC, p));
    }
    std::optional<Handle> createSliderJoint(const SliderJointConstraintSystem::CreateParams& p)
    {
        return create(axisJoint(AG2D_JOINT_SLIDER, p));
    }
    std::optional<Handle> createMotor(const MotorConstraintSystem::CreateParams& p)
    {
        ag2d_joint_desc d{};
        d.kind = AG2D_JOINT_MOTOR;
        d.body_a = p.bodyHandle.value;
        d.target_speed = p.targetSpeed; d.max_torque = p.maxTorque;
        return create(d);
    }
    void destroySpring(Handle h) { destroy(AG2D_JOINT_SPRING, h); }
    void destroyRevoluteJoint(Handle h) { destroy(AG2D_JOINT_REVOLUTE, h); }
    void destroyPrismaticJoint(Handle h) { destroy(AG2D_JOINT_PRISMATIC, h); }
    void destroySliderJoint(Handle h) { destroy(AG2D_JOINT_SLIDER, h); }
    void destroyMotor(Handle h) { destroy(AG2D_JOINT_MOTOR, h); }

    void setSpringRestLength(Handle h, Real v) { set(AG2D_JOINT_SPRING, h, AG2D_JOINT_REST_LENGTH, v); }
    void setSpringStiffness(Handle h, Real v) { set(AG2D_JOINT_SPRING, h, AG2D_JOINT_STIFFNESS, v); }
    void setSpringDamping(Handle h, Real v) { set(AG2D_JOINT_SPRING, h, AG2D_JOINT_DAMPING, v); }
    void setRevoluteJointStiffness(Handle h, Real v) { set(AG2D_JOINT_REVOLUTE, h, AG2D_JOINT_STIFFNESS, v); }
    void setRevoluteJointDamping(Handle h, Real v) { set(AG2D_JOINT_REVOLUTE, h, AG2D_JOINT_DAMPING, v); }
    void setPrismaticJointLimits(Handle h, Real lower, Real upper)
    {
        set(AG2D_JOINT_PRISMATIC, h, AG2D_JOINT_LIMITS, lower, upper);
    }
    void setPrismaticJointEnableLimit(Handle h, bool e) { set(AG2D_JOINT_PRISMATIC, h, AG2D_JOINT_ENABLE_LIMIT, e); }
    void resetPrismaticJointReferenceAngle(Handle h) { set(AG2D_JOINT_PRISMATIC, h, AG2D_JOINT_RESET_REFERENCE_ANGLE, 0); }
    void setSliderJointLimits(Handle h, Real lower, Real upper)
    {
        set(AG2D_JOINT_SLIDER, h, AG2D_JOINT_LIMITS, lower, upper);
    }
    void setSliderJointEnableLimit(Handle h, bool e) { set(AG2D_JOINT_SLIDER, h, AG2D_JOINT_ENABLE_LIMIT, e); }
    void setMotorTargetSpeed(Handle h, Real v) { set(AG2D_JOINT_MOTOR, h, AG2D_JOINT_TARGET_SPEED, v); }
    void setMotorMaxTorque(Handle h, Real v) { set(AG2D_JOINT_MOTOR, h, AG2D_JOINT_MAX_TORQUE, v); }

    // The constraint as stored now (get*DataH); nullopt if stale. The motor's accumulated impulse is in 'impulse'.
    std::optional<ag2d_joint_desc> getData(int32_t kind, Handle h) const
    {
        ag2d_joint_desc d{};
        if (ag2d_world_joint(world, kind, h.value, &d) != AG2D_OK) return std::nullopt;
        return d;
    }

private:
    static ag2d_joint_desc pair(int32_t kind, Handle a, Handle b, Vec2 anchorA, Vec2 anchorB)
    {
        ag2d_joint_desc d{};
        d.kind = kind;
        d.body_a = a.value; d.body_b = b.value;
        d.anchor_a_x = anchorA.x; d.anchor_a_y = anchorA.y; d.anchor_b_x = anchorB.x; d.anchor_b_y = anchorB.y;
        return d;
    }
    static ag2d_joint_desc axisJoint(int32_t kind, const PrismaticJointConstraintSystem::CreateParams& p)
    {
        ag2d_joint_desc d = pair(kind, p.bodyHandleA, p.bodyHandleB, p.localAnchorA, p.localAnchorB);
        d.axis_x = p.localAxisA.x; d.axis_y = p.localAxisA.y;
        d.stiffness = p.stiffness; d.damping = p.damping;
        d.lower_limit = p.lowerLimit; d.upper_limit = p.upperLimit; d.enable_limit = p.enableLimit ? 1 : 0;
        return d;
    }
    std::optional<Handle> create(const ag2d_joint_desc& d)
    {
        uint64_t h = 0;
        const int32_t rc = ag2d_world_create_joint(world, &d, &h);
        if (rc == AG2D_ERR_INVALID_ARG) return std::nullopt;
        detail::check(rc);
        return Handle{h};
    }
    void destroy(int32_t kind, Handle h) { detail::check(ag2d_world_destroy_joint(world, kind, h.value)); }
    void set(int32_t kind, Handle h, int32_t field, Real a, Real b = 0)
    {
        detail::check(ag2d_world_set_joint(world, kind, h.value, field, a, b));
    }
    ag2d_world* world;
};

class Simulation {
public:
    explicit Simulation(const SimulationSettings& s = {}) : settings(s)
    {
        ag2d_world_settings w{};
        w.dt = s.clockSettings.updateInterval * s.clockSettings.timeScale;
        w.velocity_iterations = s.collisionVelocitySolvingIterations;
        w.position_iterations = s.collisionPositionSolvingIterations;
        w.gravity_x = s.integratorSettings.gravity.x;
        w.gravity_y = s.integratorSettings.gravity.y;
        w.angular_damping = s.integratorSettings.angularVelocityDamping;
        w.sleep_speed = s.sleepSpeedThreshold;
        w.sleep_time = s.sleepTimeThreshold;
        w.ccd = s.continuousCollisionEnabled ? 1 : 0;
        w.device = s.device;
        detail::check(ag2d_world_create(&w, &world));
        api = std::make_unique<ObjectAPI>(world);
        constraintApi = std::make_unique<ConstraintAPI>(world);
    }
    ~Simulation() { ag2d_world_destroy(world); }
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;

    // Simulation::update (Simulation.cpp:32-74) with FixedClock::advance (FixedClock.h:35-63): the call's time,
    // capped at maxDeltaTimePerUpdateCall, accumulates; every whole updateInterval in the accumulator is one step.
    void update(Real deltaTime)
    {
        if (!(deltaTime > 0)) return;
        detail::check(ag2d_world_set_collision_events(world, settings.collisionEventsEnabled ? 1 : 0));
        accumulator += std::fmin(deltaTime, settings.clockSettings.maxDeltaTimePerUpdateCall);
        const uint32_t steps = uint32_t(std::floor(accumulator / settings.clockSettings.updateInterval));
        accumulator -= Real(steps) * settings.clockSettings.updateInterval;
        if (steps) detail::check(ag2d_world_step(world, int32_t(steps)));
    }

    MaterialIndex createMaterial(const Material& m)
    {
        uint32_t idx = 0;
        detail::check(ag2d_world_add_material(world, m.elasticity, m.staticFriction, m.dynamicFriction, &idx));
        return idx;
    }

    ObjectAPI& objects() noexcept { return *api; }
    // Simulation::constraints (Simulation.h:201-202).
    ConstraintAPI& constraints() noexcept { return *constraintApi; }
    const ObjectAPI& objects() const noexcept { return *api; }

    // The manifolds of the last step (Simulation::getBodyCollisionData, Simulation.h:186), as host copies.
    std::vector<ag2d_manifold> getBodyCollisionData() const
    {
        uint64_t bytes = 0;
        detail::check(ag2d_world_read(world, AG2D_PREV_MANIFOLDS, nullptr, 0, &bytes));
        std::vector<ag2d_manifold> m(bytes / sizeof(ag2d_manifold));
        detail::check(ag2d_world_read(world, AG2D_PREV_MANIFOLDS, m.data(), bytes, &bytes));
        return m;
    }

    const SimulationSettings& getSimulationSettings() const noexcept { return settings; }
    // collisionEventsEnabled is read at every update; the other fields when the Simulation is constructed.
    SimulationSettings& getSimulationSettings() noexcept { return settings; }

    // Collision callbacks (Simulation.h:169-179): fired after each step, per collider side, when a manifold's
    // impact impulse reaches the collider's threshold. nullopt for a null function or a full table.
    std::optional<CollisionCallbackIndex> createCollisionCallback(CollisionCallback function, void* userData = nullptr)
    {
        if (!function) return std::nullopt;
        auto entry = std::make_unique<CallbackEntry>(CallbackEntry{this, function, userData});
        uint16_t id = 0;
        const int32_t rc = ag2d_world_create_collision_callback(world, &Simulation::dispatch, entry.get(), &id);
        if (rc == AG2D_ERR_CAPACITY) return std::nullopt;
        detail::check(rc);
        callbackEntries[id] = std::move(entry);
        return id;
    }
    // Colliders using it are reset to no callback. false for id 0 and dead ids.
    bool destroyCollisionCallback(CollisionCallbackIndex callbackIndex)
    {
        if (ag2d_world_destroy_collision_callback(world, callbackIndex) != AG2D_OK) return false;
        callbackEntries.erase(callbackIndex);
        return true;
    }
    // Id 0 clears the collider's callback (threshold ignored). false for an invalid collider, a dead id, or a
    // negative threshold.
    bool setColliderCollisionCallback(ObjectDenseIndex colliderIndex, CollisionCallbackIndex callbackIndex,
                                      Real impulseThreshold)
    {
        return ag2d_world_set_collider_collision_callback(world, colliderIndex, callbackIndex, impulseThreshold) ==
               AG2D_OK;
    }
    // The last step's events in dispatch order (BodyCollisionSolver::getCollisionEvents, BodyCollisionSolver.h:125).
    std::vector<CollisionEvent> getCollisionEvents() const
    {
        uint32_t n = 0;
        detail::check(ag2d_world_collision_events(world, nullptr, 0, &n));
        std::vector<ag2d_collision_event> raw(n);
        if (n) detail::check(ag2d_world_collision_events(world, raw.data(), n, &n));
        std::vector<CollisionEvent> out;
        out.reserve(raw.size());
        for (const ag2d_collision_event& e : raw) out.push_back(convert(e));
        return out;
    }
    // Simulation::getBroadPhaseCollisionDetector / getNarrowPhaseCollisionDetector (Simulation.h:183-184), for their
    // query entry points.
    BroadPhaseCollisionDetector getBroadPhaseCollisionDetector() const noexcept { return BroadPhaseCollisionDetector(world); }
    NarrowPhaseCollisionDetector getNarrowPhaseCollisionDetector() const noexcept { return NarrowPhaseCollisionDetector(world); }
    ag2d_world* handle() noexcept { return world; }

private:
    struct CallbackEntry {
        Simulation* sim;
        CollisionCallback fn;
        void* user;
    };
    static CollisionEvent convert(const ag2d_collision_event& e)
    {
        CollisionEvent ev;
        ev.self = e.self;
        ev.other = e.other;
        ev.selfBody = Handle{e.self_body_handle};
        ev.otherBody = Handle{e.other_body_handle};
        ev.point = Vec2{e.point_x, e.point_y};
        ev.normal = Vec2{e.normal_x, e.normal_y};
        ev.impulse = e.impulse;
        ev.callbackId = e.callback_id;
        return ev;
    }
    // The C callback of every id: the entry is copied first, so the user function may destroy its own id.
    static void dispatch(const ag2d_collision_event* e, ag2d_world*, void* user)
    {
        const CallbackEntry entry = *static_cast<const CallbackEntry*>(user);
        entry.fn(convert(*e), *entry.sim, entry.user);
    }

    SimulationSettings settings;
    ag2d_world* world = nullptr;
    std::unique_ptr<ObjectAPI> api;
    std::unique_ptr<ConstraintAPI> constraintApi;
    Real accumulator = 0;
    std::map<CollisionCallbackIndex, std::unique_ptr<CallbackEntry>> callbackEntries;
};

}  // namespace ag2d
