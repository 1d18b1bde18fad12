// Scene code in the reference's style (App/Scenes.cpp: create a material, a static ground box and a pile of
// bodies through ObjectAPI, then Simulation::update) compiled against the C++ facade of libag2d.so.
// Prints "no-device" and exits 0 when the machine has no CUDA device; otherwise steps the scene (a capsule is
// created among the pile, and a body with three colliders; once it has settled one body is destroyed and another
// kicked upwards through ObjectAPI's deferred commands) and prints "ok <bodies> <most manifolds in one step> <mean y>
// <colliders a circle query finds> <circle contacts> <colliders in the trees> <impacts on the ground> <largest
// impact impulse>" after querying the settled pile the way the reference's editor selects
// (queryCollidersInShape with a CircleQuery, then findCollisionsInCircle over what it found).
#include "ag2d_simulation.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>

int main()
{
    ag2d::SimulationSettings settings;
    settings.clockSettings.updateInterval = 1.0f / 60.0f;
    settings.collisionVelocitySolvingIterations = 8;
    std::optional<ag2d::Simulation> sim;
    try {
        sim.emplace(settings);
    } catch (const std::runtime_error& e) {
        if (std::strstr(e.what(), "no CUDA device")) { std::printf("no-device\n"); return 0; }
        std::printf("error %s\n", e.what());
        return 1;
    }
    const ag2d::MaterialIndex mat = sim->createMaterial({0.0f, 0.4f, 0.4f});
    ag2d::BoxCreateParams ground;
    ground.base.position = {0.0f, -1.0f};
    ground.base.materialIndex = mat;
    ground.size = {40.0f, 2.0f};
    if (!sim->objects().createBox(ground)) return 2;
    // Impacts on the ground (its collider is the first): counted by a collision callback.
    struct Impacts { int count = 0; ag2d::Real largest = 0; } impacts;
    const auto onImpact = [](const ag2d::CollisionEvent& e, ag2d::Simulation&, void* user) {
        auto* im = static_cast<Impacts*>(user);
        im->count++;
        im->largest = std::max(im->largest, e.impulse);
    };
    const std::optional<ag2d::CollisionCallbackIndex> impactId = sim->createCollisionCallback(onImpact, &impacts);
    if (!impactId || !sim->setColliderCollisionCallback(0, *impactId, 0.5f)) return 14;
    if (sim->setColliderCollisionCallback(0, *impactId, -1.0f)) return 15;   // negative threshold: false
    ag2d::Vec2 tri[3] = {{-0.5f, -0.4f}, {0.5f, -0.4f}, {0.0f, 0.6f}};
    int created = 1;
    for (int i = 0; i < 60; i++) {
        ag2d::BodyCreateParams b;
        b.position = {-12.0f + float(i % 12) * 2.0f, 1.0f + float(i / 12) * 1.5f};
        b.mass = 1.0f;
        b.materialIndex = mat;
        bool ok;
        if (i % 3 == 0) ok = sim->objects().createCircle({b, 0.45f}).has_value();
        else if (i % 3 == 1) ok = sim->objects().createBox({b, {0.8f, 0.8f}}).has_value();
        else ok = sim->objects().createPolygon({b, std::span<ag2d::Vec2>(tri, 3)}).has_value();
        created += ok ? 1 : 0;
    }
    // ObjectAPI::setPolygonShape on the first triangle's collider: a square is queued, a concave dart refused.
    ag2d::Vec2 square[4] = {{-0.4f, -0.4f}, {0.4f, -0.4f}, {0.4f, 0.4f}, {-0.4f, 0.4f}};
    ag2d::Vec2 dart[4] = {{0.0f, 0.0f}, {1.0f, 0.5f}, {0.0f, 0.2f}, {-1.0f, 0.5f}};
    if (!sim->objects().setPolygonShape(3, square) || sim->objects().setPolygonShape(3, dart)) return 40;
    ag2d::BodyCreateParams cb;
    cb.position = {0.0f, 10.0f};
    cb.rotation = 0.3f;
    cb.mass = 1.0f;
    cb.materialIndex = mat;
    const std::optional<ag2d::Handle> capsule = sim->objects().createCapsuleH({cb, 1.5f, 0.3f});
    if (!capsule) return 7;
    created++;
    ag2d::BodyCreateParams gb;
    gb.position = {8.0f, 10.0f};
    gb.mass = 1.0f;
    gb.materialIndex = mat;
    const std::optional<ag2d::Handle> doomed = sim->objects().createCircleH({gb, 0.5f});
    if (!doomed) return 8;
    created++;
    // A compound body (ObjectAPI::createBody + create*Collider): a bar with a wheel at each end, and an invalid
    // collider request on a stale handle.
    ag2d::BodyCreateParams db;
    db.position = {-4.0f, 12.0f};
    db.mass = 2.0f;
    db.inertia = 1.5f;
    const std::optional<ag2d::Handle> dumbbell = sim->objects().createBodyH(db);
    if (!dumbbell) return 10;
    created++;
    ag2d::BoxColliderCreateParams bar;
    bar.bodyHandle = *dumbbell;
    bar.materialIndex = mat;
    bar.size = {2.0f, 0.2f};
    if (!sim->objects().createBoxCollider(bar)) return 11;
    for (float side : {-1.0f, 1.0f}) {
        ag2d::CircleColliderCreateParams wheel;
        wheel.bodyHandle = *dumbbell;
        wheel.localOffset = {side, 0.0f};
        wheel.materialIndex = mat;
        wheel.radius = 0.35f;
        if (!sim->objects().createCircleCollider(wheel)) return 12;
    }
    // A concave bracket on the bar: split into convex pieces, one collider each.
    ag2d::Vec2 bracket[6] = {{-0.6f, 0.1f}, {0.6f, 0.1f}, {0.6f, 0.7f}, {0.4f, 0.7f}, {0.4f, 0.3f}, {-0.6f, 0.3f}};
    ag2d::PolygonColliderCreateParams bracketParams;
    bracketParams.bodyHandle = *dumbbell;
    bracketParams.materialIndex = mat;
    bracketParams.localVertices = std::span<const ag2d::Vec2>(bracket, 6);
    const auto pieces = sim->objects().createPolygonCollider(bracketParams);
    if (!pieces || pieces->colliderCount < 2) return 41;
    // A swinging chain (ConstraintAPI): three links on revolute joints from a static hook, a motor on the last.
    ag2d::BodyCreateParams hb;
    hb.position = {14.0f, 14.0f};
    const std::optional<ag2d::Handle> hook = sim->objects().createBodyH(hb);
    if (!hook) return 16;
    created++;
    ag2d::Handle prevLink = *hook;
    for (int k = 0; k < 3; k++) {
        ag2d::BodyCreateParams lb;
        lb.position = {15.0f + float(k), 14.0f};
        lb.mass = 1.0f;
        lb.inertia = 0.1f;
        const std::optional<ag2d::Handle> link = sim->objects().createBodyH(lb);
        if (!link) return 17;
        created++;
        ag2d::RevoluteJointConstraintSystem::CreateParams jp;
        jp.bodyHandleA = prevLink;
        jp.bodyHandleB = *link;
        jp.localAnchorA = {k == 0 ? 0.0f : 0.5f, 0.0f};
        jp.localAnchorB = {-0.5f, 0.0f};
        jp.stiffness = 1.0e4f;
        jp.damping = 20.0f;
        if (!sim->constraints().createRevoluteJoint(jp)) return 18;
        prevLink = *link;
    }
    if (!sim->constraints().createMotor({prevLink, 3.0f, 10.0f})) return 19;
    if (sim->constraints().createMotor({ag2d::Handle{~0ull}, 1.0f, 1.0f})) return 20;   // stale body: nullopt
    ag2d::CircleColliderCreateParams orphan;
    orphan.bodyHandle = ag2d::Handle{~0ull};
    orphan.radius = 1.0f;
    if (sim->objects().createCircleCollider(orphan)) return 13;   // stale body handle: nullopt
    ag2d::BoxCreateParams bad;
    bad.base.mass = 1.0f;
    bad.size = {-1.0f, 1.0f};
    if (sim->objects().createBox(bad)) return 3;     // invalid shape: nullopt, as in the reference
    size_t maxManifolds = 0;   // the pile settles and falls asleep, so track the most contacts seen
    for (int frame = 0; frame < 120; frame++) {
        if (frame == 90) {
            sim->objects().destroyBody(*doomed);
            sim->objects().setBodyVelocity(*capsule, {0.0f, 3.0f});
        }
        sim->update(1.0f / 60.0f);
        maxManifolds = std::max(maxManifolds, sim->getBodyCollisionData().size());
    }
    if (sim->objects().getBodyIndex(*doomed) != UINT32_MAX) return 9;   // the destroyed body's handle is stale
    const ag2d::BodyView bodies = sim->objects().getBodies();
    double meanY = 0.0;
    for (uint32_t i = 0; i < bodies.getCount(); i++) meanY += bodies.comY[i];
    namespace bp = ag2d::BroadPhaseInternal;
    std::vector<ag2d::ObjectDenseIndex> found;
    sim->getBroadPhaseCollisionDetector().queryCollidersInShape(bp::CircleQuery({0.0f, 1.0f}, 3.0f),
                                                                bp::BvhTreeTypeFlag::All, found);
    std::vector<std::pair<ag2d::ObjectDenseIndex, ag2d::Real>> touching;
    sim->getNarrowPhaseCollisionDetector().findCollisionsInCircle(found, {0.0f, 1.0f}, 3.0f, touching);
    for (const auto& t : touching)
        if (!(t.second < 3.0f)) return 5;   // a contact is closer than the radius
    // A collidersToCheck that is not a circle query's output (every other one of them): exactly the full answer's
    // contacts among those colliders.
    std::vector<ag2d::ObjectDenseIndex> half;
    for (size_t i = 0; i < found.size(); i += 2) half.push_back(found[i]);
    std::vector<std::pair<ag2d::ObjectDenseIndex, ag2d::Real>> touchingHalf;
    sim->getNarrowPhaseCollisionDetector().findCollisionsInCircle(half, {0.0f, 1.0f}, 3.0f, touchingHalf);
    {
        size_t expect = 0;
        for (const auto& t : touching)
            if (std::find(half.begin(), half.end(), t.first) != half.end()) expect++;
        if (touchingHalf.size() != expect) return 21;
        for (const auto& t : touchingHalf)
            if (std::find(half.begin(), half.end(), t.first) == half.end()) return 22;
    }
    std::vector<ag2d::ObjectDenseIndex> all;
    sim->getBroadPhaseCollisionDetector().queryCollidersInShape(bp::AABBQuery({-1e6f, -1e6f, 1e6f, 1e6f}),
                                                                bp::BvhTreeTypeFlag::All, all);
    // One collider per live body plus the dumbbell's two wheels and the bracket's pieces, all inside the huge box;
    // the destroyed body's collider is in no tree, and the hook and the chain's three links have none.
    if (all.size() != bodies.getCount() - 1 + 2 - 4 + pieces->colliderCount) {
        std::printf("colliders found %zu, bodies %u\n", all.size(), bodies.getCount());
        return 6;
    }
    std::printf("ok %u %zu %.3f %zu %zu %zu %d %.3f\n", bodies.getCount(), maxManifolds,
                meanY / double(bodies.getCount()), found.size(), touching.size(), all.size(), impacts.count,
                double(impacts.largest));
    return bodies.getCount() == uint32_t(created) ? 0 : 4;
}
