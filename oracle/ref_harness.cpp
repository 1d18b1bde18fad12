// Test harness around the reference engine (PS_AGONY2D) compiled on the CPU.
//
// TEST INFRASTRUCTURE ONLY. It is linked into oracle/_ref/libagony_ref.so by oracle/ref_build.sh and is loaded by
// tests/golden/make_golden.py (golden vectors), by the oracle self-checks in tests/, and by bench.py's reference arm
// (the timed CPU baseline). Nothing in the product path loads it.
//
// The harness drives the reference's own public API (Simulation::update, ObjectAPI::create*, createMaterial) and,
// for per-phase golden vectors, the same member functions Simulation::physicsStep calls
// (PhysicsSimulation-Agony/PS_AGONY2D/Simulation.cpp:255-351), reading intermediate state in between. Private
// members are reached by compiling this file with -fno-access-control.
#include "PS_AGONY2D/Simulation.h"
#include "PS_AGONY2D/FastCosSin.h"
#include "PS_AGONY2D/Threading.h"
#include "PS_AGONY2D/SimulationImpl/LeftOutFunctions.h"
#include "PS_AGONY2D/SimulationImpl/PhysicsGeometry.h"
#include "PS_AGONY2D/SimulationImpl/PolygonDecomposition.h"

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

using namespace PS_AGONY2D;

namespace
{
    // IThreadingBackend (PS_AGONY2D/Threading.h:10-22): every launched task runs on its own pool thread, all
    // concurrently, and launch() returns without waiting — the contract the reference's wave runner relies on.
    class PoolBackend final : public Threading::IThreadingBackend
    {
        struct Worker
        {
            std::thread thread;
            std::mutex m;
            std::condition_variable cv;
            Threading::TaskFn fn = nullptr;
            void* ctx = nullptr;
            size_t index = 0;
            bool has = false;
            bool stop = false;
        };
        std::vector<std::unique_ptr<Worker>> workers;

    public:
        explicit PoolBackend(size_t threads)
        {
            for (size_t i = 0; i < threads; i++)
            {
                workers.emplace_back(std::make_unique<Worker>());
                Worker* w = workers.back().get();
                w->thread = std::thread([w] {
                    for (;;)
                    {
                        Threading::TaskFn fn;
                        void* ctx;
                        size_t index;
                        {
                            std::unique_lock<std::mutex> lk(w->m);
                            w->cv.wait(lk, [w] { return w->has || w->stop; });
                            if (w->stop && !w->has) return;
                            fn = w->fn; ctx = w->ctx; index = w->index;
                        }
                        fn(ctx, index);
                        {
                            std::lock_guard<std::mutex> lk(w->m);
                            w->has = false;
                        }
                        w->cv.notify_all();
                    }
                });
            }
        }
        ~PoolBackend() override
        {
            for (auto& w : workers)
            {
                {
                    std::unique_lock<std::mutex> lk(w->m);
                    w->cv.wait(lk, [&] { return !w->has; });
                    w->stop = true;
                }
                w->cv.notify_all();
                w->thread.join();
            }
        }
        size_t getThreadCount() const noexcept override { return workers.size(); }
        void launch(size_t taskCount, Threading::TaskFn fn, void* context, std::span<const uint32_t>) override
        {
            for (size_t i = 0; i < taskCount; i++)
            {
                Worker* w = workers[i % workers.size()].get();
                std::unique_lock<std::mutex> lk(w->m);
                w->cv.wait(lk, [w] { return !w->has; }); // Previous task on this worker finished.
                w->fn = fn; w->ctx = context; w->index = i; w->has = true;
                lk.unlock();
                w->cv.notify_all();
            }
        }
    };

    std::mutex g_backendMutex;
    std::map<size_t, std::unique_ptr<PoolBackend>> g_backends;

    PoolBackend* backendFor(size_t threads)
    {
        std::lock_guard<std::mutex> lk(g_backendMutex);
        auto& b = g_backends[threads];
        if (!b) b = std::make_unique<PoolBackend>(threads);
        return b.get();
    }

    struct Harness
    {
        Simulation sim;
        float dt = 1.0f / 60.0f;
        size_t threads = 0;
        std::map<std::string, std::vector<uint8_t>> blobs;
        std::vector<uint32_t> createdGeneration;   // per body handle slot: its generation when the body was created
        // Collision events the recording callback received (Types/CollisionEvent.h:18-26), by handle slots.
        struct Event
        {
            uint32_t self, other, selfBody, otherBody, callback;
            float px, py, nx, ny, impulse;
        };
        std::vector<Event> events;

        template <class T>
        void put(const std::string& name, const T* data, size_t count)
        {
            auto& b = blobs[name];
            b.resize(count * sizeof(T));
            if (count) std::memcpy(b.data(), data, count * sizeof(T));
        }
        template <class V>
        void putv(const std::string& name, const V& v) { put(name, v.data(), v.size()); }
    };

    void useBackend(Harness* h)
    {
        Threading::setThreadingBackend(backendFor(h->threads));
    }

    void dumpBodies(Harness* h, const std::string& p)
    {
        const BodySoA& b = h->sim.objectManager.bodies;
        h->putv(p + "body.comX", b.comX);
        h->putv(p + "body.comY", b.comY);
        h->putv(p + "body.velocityX", b.velocityX);
        h->putv(p + "body.velocityY", b.velocityY);
        h->putv(p + "body.rotation", b.rotation);
        h->putv(p + "body.angularVelocity", b.angularVelocity);
        h->putv(p + "body.mass", b.mass);
        h->putv(p + "body.invMass", b.invMass);
        h->putv(p + "body.inertia", b.inertia);
        h->putv(p + "body.invInertia", b.invInertia);
        h->putv(p + "body.rotationCos", b.rotationCos);
        h->putv(p + "body.rotationSin", b.rotationSin);
        h->putv(p + "body.boundRadius", b.boundRadius);
        h->putv(p + "body.sleepingTimer", b.sleepingTimer);
        h->putv(p + "body.renderRotationWrapCount", b.renderRotationWrapCount);
        h->putv(p + "body.localCenterOfMassX", b.localCenterOfMassX);
        h->putv(p + "body.localCenterOfMassY", b.localCenterOfMassY);
        h->putv(p + "body.islandId", b.islandId);
        h->putv(p + "body.sleepIslandId", b.sleepIslandId);
        h->put(p + "body.groupStarts", b.groupStarts, size_t(BodyGroup::Unused) + 1);
        std::vector<uint32_t> slot(b.getCount()), gen(b.getCount());
        for (size_t i = 0; i < b.getCount(); i++)
        {
            const Handle hd = b.handleAt(uint32_t(i));
            slot[i] = hd.slot; gen[i] = hd.generation;
        }
        h->putv(p + "body.handleSlot", slot);
        h->putv(p + "body.handleGen", gen);
    }

    void dumpColliders(Harness* h, const std::string& p)
    {
        const ObjectManager& om = h->sim.objectManager;
        const ColliderSoA& c = om.colliders;
        h->putv(p + "col.bodyIndex", c.bodyIndex);
        h->putv(p + "col.localOffsetX", c.localOffsetX);
        h->putv(p + "col.localOffsetY", c.localOffsetY);
        h->putv(p + "col.comOffsetX", c.comOffsetX);
        h->putv(p + "col.comOffsetY", c.comOffsetY);
        h->putv(p + "col.localRotation", c.localRotation);
        h->putv(p + "col.worldPosX", c.worldPosX);
        h->putv(p + "col.worldPosY", c.worldPosY);
        h->putv(p + "col.worldRotation", c.worldRotation);
        h->putv(p + "col.worldRotationCos", c.worldRotationCos);
        h->putv(p + "col.worldRotationSin", c.worldRotationSin);
        h->putv(p + "col.materialIndex", c.materialIndex);
        std::vector<uint32_t> st(c.getCount());
        for (size_t i = 0; i < c.getCount(); i++) st[i] = uint32_t(c.shapeType[i]);
        h->putv(p + "col.shapeType", st);
        h->putv(p + "col.shapeIndex", c.shapeIndex);
        h->putv(p + "col.aabbMinX", c.aabbMinX);
        h->putv(p + "col.aabbMinY", c.aabbMinY);
        h->putv(p + "col.aabbMaxX", c.aabbMaxX);
        h->putv(p + "col.aabbMaxY", c.aabbMaxY);
        h->putv(p + "col.minExtent", c.minExtent);
        h->putv(p + "col.maxExtent", c.maxExtent);
        h->put(p + "col.groupStarts", c.groups.starts, size_t(BodyGroup::Unused) + 1);
        std::vector<uint32_t> slot(c.getCount()), gen(c.getCount());
        for (size_t i = 0; i < c.getCount(); i++)
        {
            const Handle hd = c.handleAt(uint32_t(i));
            slot[i] = hd.slot; gen[i] = hd.generation;
        }
        h->putv(p + "col.handleSlot", slot);
        h->putv(p + "col.handleGen", gen);
        std::vector<uint32_t> cb(c.getCount());
        for (size_t i = 0; i < c.getCount(); i++) cb[i] = uint32_t(c.callbackId[i]);
        h->putv(p + "col.callbackId", cb);
        h->putv(p + "col.eventThreshold", c.eventThreshold);

        h->putv(p + "circle.colliderIndices", om.circles.colliderIndices);
        h->putv(p + "circle.radius", om.circles.radius);
        h->putv(p + "box.colliderIndices", om.boxes.colliderIndices);
        h->putv(p + "box.halfWidth", om.boxes.halfWidth);
        h->putv(p + "box.halfHeight", om.boxes.halfHeight);
        h->putv(p + "poly.colliderIndices", om.polygons.colliderIndices);
        std::vector<uint32_t> counts;
        std::vector<float> verts, norms;
        for (const PolygonGeometry& g : om.polygons.geometry)
        {
            counts.push_back(uint32_t(g.size()));
            for (size_t v = 0; v < g.size(); v++)
            {
                verts.push_back(g.vertices()[v].x); verts.push_back(g.vertices()[v].y);
                norms.push_back(g.normals()[v].x); norms.push_back(g.normals()[v].y);
            }
        }
        h->putv(p + "poly.counts", counts);
        h->putv(p + "poly.vertices", verts);
        h->putv(p + "poly.normals", norms);
        h->putv(p + "capsule.colliderIndices", om.capsules.colliderIndices);
        h->putv(p + "capsule.halfLength", om.capsules.halfLength);
        h->putv(p + "capsule.radius", om.capsules.radius);
    }

    // Manifolds with collider handles resolved to current dense collider indices.
    void dumpManifolds(Harness* h, const std::string& p, std::span<const BodyCollisionData> m)
    {
        const HandleTable& handles = h->sim.objectManager.colliders.handles;
        std::vector<uint32_t> a(m.size()), b(m.size()), aslot(m.size()), bslot(m.size()), cnt(m.size()), ids(2 * m.size());
        std::vector<float> nrm(2 * m.size()), depth(m.size()), pts(4 * m.size()), imp(4 * m.size());
        for (size_t i = 0; i < m.size(); i++)
        {
            const BodyCollisionData& d = m[i];
            a[i] = handles.indexOf(d.colliderA);
            b[i] = handles.indexOf(d.colliderB);
            aslot[i] = d.colliderA.slot;
            bslot[i] = d.colliderB.slot;
            cnt[i] = d.contactCount;
            nrm[2 * i] = d.normal.x; nrm[2 * i + 1] = d.normal.y;
            depth[i] = d.penetration;
            for (int k = 0; k < 2; k++)
            {
                const bool live = uint32_t(k) < d.contactCount;
                pts[4 * i + 2 * k] = live ? d.contactPoints[k].x : 0.0f;
                pts[4 * i + 2 * k + 1] = live ? d.contactPoints[k].y : 0.0f;
                ids[2 * i + k] = live ? d.contactIds[k] : 0u;
                imp[4 * i + 2 * k] = d.persistentContactData[k].normalImpulseAccumulator;
                imp[4 * i + 2 * k + 1] = d.persistentContactData[k].tangentImpulseAccumulator;
            }
        }
        h->putv(p + "colA", a); h->putv(p + "colB", b);
        h->putv(p + "slotA", aslot); h->putv(p + "slotB", bslot);
        h->putv(p + "count", cnt); h->putv(p + "normal", nrm); h->putv(p + "depth", depth);
        h->putv(p + "points", pts); h->putv(p + "ids", ids); h->putv(p + "impulses", imp);
    }

    // The sleeping islands' stored manifolds (NarrowPhaseCollisionDetector::islandManifolds), flattened in island
    // slot order, with each record's sleep island id (slot + FIRST_SLEEP_ISLAND_ID) as <p>islandId.
    void dumpIslandStore(Harness* h, const std::string& p)
    {
        const auto& store = h->sim.narrowPhaseCollisionDetector.islandManifolds;
        std::vector<BodyCollisionData> flat;
        std::vector<uint32_t> id;
        for (size_t slot = 0; slot < store.size(); slot++)
            for (const BodyCollisionData& d : store[slot]) {
                flat.push_back(d);
                id.push_back(uint32_t(slot + FIRST_SLEEP_ISLAND_ID));
            }
        dumpManifolds(h, p, flat);
        h->putv(p + "islandId", id);
    }

    void dumpTree(Harness* h, const std::string& p, BroadPhaseInternal::BvhTreeType type)
    {
        const auto& t = h->sim.broadPhaseCollisionDetector.trees[size_t(type)];
        h->putv(p + "sorted", t.colliderIndices);
        h->putv(p + "morton", t.mortonCodes);
    }

    int64_t finishBody(Harness* h, std::optional<ObjectDenseIndex> idx)
    {
        if (!idx) return -1;
        const Handle hd = h->sim.objectManager.bodies.handleAt(*idx);
        if (h->createdGeneration.size() <= hd.slot) h->createdGeneration.resize(size_t(hd.slot) + 1, 0u);
        h->createdGeneration[hd.slot] = hd.generation;
        return int64_t(hd.slot);
    }
}

extern "C"
{
    struct agref_settings
    {
        float dt;
        uint32_t velocity_iterations;
        uint32_t position_iterations;
        float gravity_x, gravity_y;
        int32_t ccd;
        float sleep_speed;
        float sleep_time;
        int32_t threads; // Pool threads besides the calling one (0 = single-threaded).
    };

    void* agref_create(const agref_settings* s)
    {
        auto* h = new Harness();
        h->dt = s->dt;
        h->threads = size_t(s->threads < 0 ? 0 : s->threads);
        auto& ss = h->sim.getSimulationSettings();
        ss.clockSettings.updateInterval = s->dt;
        ss.collisionVelocitySolvingIterations = s->velocity_iterations;
        ss.collisionPositionSolvingIterations = s->position_iterations;
        ss.integratorSettings.gravity = Vec2(s->gravity_x, s->gravity_y);
        ss.continuousCollisionEnabled = s->ccd != 0;
        ss.sleepSpeedThreshold = s->sleep_speed;
        ss.sleepTimeThreshold = s->sleep_time;
        return h;
    }

    void agref_destroy(void* hp) { delete static_cast<Harness*>(hp); }

    uint32_t agref_material(void* hp, float elasticity, float staticFriction, float dynamicFriction)
    {
        Material m;
        m.elasticity = elasticity; m.staticFriction = staticFriction; m.dynamicFriction = dynamicFriction;
        return static_cast<Harness*>(hp)->sim.createMaterial(m);
    }

    static BodyCreateParams baseParams(float px, float py, float rot, float vx, float vy, float w, float mass, uint32_t mat)
    {
        BodyCreateParams b;
        b.position = Vec2(px, py);
        b.velocity = Vec2(vx, vy);
        b.rotation = rot;
        b.angularVelocity = w;
        b.mass = mass;
        b.materialIndex = mat;
        return b;
    }

    // Returns the body handle slot (stable id), or -1 on failure.
    int64_t agref_add_polygon(void* hp, const float* xy, uint32_t n, float px, float py, float rot, float vx, float vy,
                              float w, float mass, uint32_t mat)
    {
        auto* h = static_cast<Harness*>(hp);
        std::vector<Vec2> v(n);
        for (uint32_t i = 0; i < n; i++) v[i] = Vec2(xy[2 * i], xy[2 * i + 1]);
        PolygonCreateParams p;
        p.base = baseParams(px, py, rot, vx, vy, w, mass, mat);
        p.localVertices = std::span<Vec2>(v.data(), v.size());
        return finishBody(h, h->sim.objects().createPolygon(p));
    }

    int64_t agref_add_box(void* hp, float width, float height, float px, float py, float rot, float vx, float vy,
                          float w, float mass, uint32_t mat)
    {
        auto* h = static_cast<Harness*>(hp);
        BoxCreateParams p;
        p.base = baseParams(px, py, rot, vx, vy, w, mass, mat);
        p.size = Vec2(width, height);
        return finishBody(h, h->sim.objects().createBox(p));
    }

    int64_t agref_add_circle(void* hp, float radius, float px, float py, float rot, float vx, float vy,
                             float w, float mass, uint32_t mat)
    {
        auto* h = static_cast<Harness*>(hp);
        CircleCreateParams p;
        p.base = baseParams(px, py, rot, vx, vy, w, mass, mat);
        p.radius = radius;
        return finishBody(h, h->sim.objects().createCircle(p));
    }

    int64_t agref_add_capsule(void* hp, float length, float radius, float px, float py, float rot, float vx,
                              float vy, float w, float mass, uint32_t mat)
    {
        auto* h = static_cast<Harness*>(hp);
        CapsuleCreateParams p;
        p.base = baseParams(px, py, rot, vx, vy, w, mass, mat);
        p.length = length;
        p.radius = radius;
        return finishBody(h, h->sim.objects().createCapsule(p));
    }

    // ObjectAPI::createBody + create*Collider (ObjectAPI.h:28-32): a body with explicit mass, inertia and centre of
    // mass, then colliders on it. Returns the body's handle slot / the collider's dense index, -1 on failure.
    int64_t agref_create_body(void* hp, float px, float py, float rot, float vx, float vy, float w, float mass,
                              float inertia, float comX, float comY)
    {
        auto* h = static_cast<Harness*>(hp);
        BodyCreateParams b = baseParams(px, py, rot, vx, vy, w, mass, 0);
        b.inertia = inertia;
        b.centerOfMass = Vec2(comX, comY);
        return finishBody(h, h->sim.objects().createBody(b));
    }
    int64_t agref_add_collider(void* hp, uint32_t slot, int32_t shape, float lx, float ly, float lrot, uint32_t mat,
                               float p0, float p1, const float* xy, uint32_t n);

    // ObjectAPI's deferred body commands (SimulationAPIs/ObjectAPI.h:72-81), by body handle slot: the handle the
    // body got at creation (so a destroyed body's handle stays stale, even once its slot is reused); the reference
    // applies them at its next flushCommands (ObjectManager.cpp:638).
    static Handle bodyHandleOfSlot(Harness* h, uint32_t slot)
    {
        return Handle{slot, slot < h->createdGeneration.size() ? h->createdGeneration[slot] : 0u};
    }
    void agref_destroy_body(void* hp, uint32_t slot)
    {
        auto* h = static_cast<Harness*>(hp);
        h->sim.objects().destroyBody(bodyHandleOfSlot(h, slot));
    }
    // kind: 0 position (a, b), 1 rotation (a), 2 velocity (a, b), 3 angular velocity (a), 4 mass (a), 5 inertia (a),
    // 6 local centre of mass (a, b), 7 recompute inertia, 8 mass from density (a).
    void agref_set_body(void* hp, uint32_t slot, int32_t kind, float a, float b)
    {
        auto* h = static_cast<Harness*>(hp);
        const Handle hd = bodyHandleOfSlot(h, slot);
        auto& o = h->sim.objects();
        switch (kind)
        {
        case 0: o.setBodyPosition(hd, Vec2(a, b)); break;
        case 1: o.setBodyRotation(hd, a); break;
        case 2: o.setBodyVelocity(hd, Vec2(a, b)); break;
        case 3: o.setBodyAngularVelocity(hd, a); break;
        case 4: o.setBodyMass(hd, a); break;
        case 5: o.setBodyInertia(hd, a); break;
        case 6: o.setBodyLocalCenterOfMass(hd, Vec2(a, b)); break;
        case 7: o.recomputeBodyInertia(hd); break;
        case 8: o.setBodyMassFromDensity(hd, a); break;
        default: break;
        }
    }
    // ObjectAPI's collider setters (SimulationAPIs/ObjectAPI.h:86-91) on the collider at a dense index now:
    // kind 0 local offset (a, b), 1 local rotation, 2 material (a), 3 circle radius, 4 box size, 5 capsule shape.
    void agref_set_collider(void* hp, uint32_t index, int32_t kind, float a, float b)
    {
        auto* h = static_cast<Harness*>(hp);
        auto& o = h->sim.objects();
        const Handle hd = h->sim.objectManager.colliders.handleAt(index);
        switch (kind)
        {
        case 0: o.setColliderLocalOffset(hd, Vec2(a, b)); break;
        case 1: o.setColliderLocalRotation(hd, a); break;
        case 2: o.setColliderMaterial(hd, MaterialIndex(a)); break;
        case 3: o.setCircleRadius(hd, a); break;
        case 4: o.setBoxSize(hd, Vec2(a, b)); break;
        case 5: o.setCapsuleShape(hd, a, b); break;
        default: break;
        }
    }
    // ObjectAPI::setPolygonShape (ObjectAPI.h:93) on the collider at dense index 'index': 1 if queued.
    int32_t agref_set_polygon(void* hp, uint32_t index, const float* xy, uint32_t n)
    {
        auto* h = static_cast<Harness*>(hp);
        const Handle hd = h->sim.objectManager.colliders.handleAt(index);
        std::vector<Vec2> v(n);
        for (uint32_t i = 0; i < n; i++) v[i] = Vec2(xy[2 * i], xy[2 * i + 1]);
        return h->sim.objects().setPolygonShape(hd, std::span<const Vec2>(v.data(), v.size())) ? 1 : 0;
    }
    // PhysicsGeometry::preparePolygonOutline + decomposeConcave (default method) + limitConvexPieceVertexCount
    // (16, default method): the pieces polygon creation makes. Returns the piece count (-1: outline refused); the
    // counts and vertices are written while they fit.
    int32_t agref_decompose(const float* xy, uint32_t n, float* out, uint32_t cap, uint32_t* counts, uint32_t pcap)
    {
        std::vector<Vec2> v(n);
        for (uint32_t i = 0; i < n; i++) v[i] = Vec2(xy[2 * i], xy[2 * i + 1]);
        auto outline = PhysicsGeometry::preparePolygonOutline(std::span<const Vec2>(v.data(), v.size()));
        if (!outline) return -1;
        auto pieces = PhysicsGeometry::decomposeConcave(*outline, PhysicsGeometry::ConcaveDecompositionMethod::Bayazit);
        PhysicsGeometry::limitConvexPieceVertexCount(pieces, MAX_POLYGON_VERTEX_COUNT,
                                                     PhysicsGeometry::ConvexDecompositionMethod::Fan);
        uint32_t at = 0;
        for (size_t k = 0; k < pieces.size(); k++) {
            if (k < pcap) counts[k] = uint32_t(pieces[k].size());
            for (const Vec2& p : pieces[k]) {
                if (at < cap) { out[2 * at] = p.x; out[2 * at + 1] = p.y; }
                at++;
            }
        }
        return int32_t(pieces.size());
    }
    // Simulation::flushCommands (Simulation.cpp:454-461) on its own: the queued commands, the wakes they cause and
    // the stored manifolds of the woken islands, as the next update would apply them first.
    void agref_flush_commands(void* hp)
    {
        static_cast<Harness*>(hp)->sim.flushCommands();
    }

    // Collision callbacks (Simulation::createCollisionCallback / setColliderCollisionCallback /
    // destroyCollisionCallback, Simulation.cpp:130-171) with one recording function: every event dispatched at the
    // end of a step (Simulation.cpp:174-180, 450) is kept until agref_dump_events.
    static void recordEvent(const CollisionEvent& e, Simulation&, void* user)
    {
        static_cast<Harness*>(user)->events.push_back(Harness::Event{
            e.self.slot, e.other.slot, e.selfBody.slot, e.otherBody.slot, uint32_t(e.callbackId),
            e.point.x, e.point.y, e.normal.x, e.normal.y, e.impulse});
    }
    int32_t agref_create_event_callback(void* hp)
    {
        auto* h = static_cast<Harness*>(hp);
        const auto id = h->sim.createCollisionCallback(&recordEvent, h);
        return id ? int32_t(*id) : -1;
    }
    int32_t agref_destroy_event_callback(void* hp, uint32_t id)
    {
        return static_cast<Harness*>(hp)->sim.destroyCollisionCallback(CollisionCallbackIndex(id)) ? 1 : 0;
    }
    int32_t agref_set_collider_callback(void* hp, uint32_t collider, uint32_t id, float threshold)
    {
        return static_cast<Harness*>(hp)->sim.setColliderCollisionCallback(collider, CollisionCallbackIndex(id),
                                                                          threshold) ? 1 : 0;
    }
    void agref_set_events_enabled(void* hp, int32_t enable)
    {
        static_cast<Harness*>(hp)->sim.getSimulationSettings().collisionEventsEnabled = enable != 0;
    }
    // The recorded events as blobs <prefix>ev.{self,other,selfBody,otherBody,callback} (handle slots, ids) and
    // ev.{px,py,nx,ny,impulse}, in dispatch order; the record is then cleared.
    void agref_dump_events(void* hp, const char* prefix)
    {
        auto* h = static_cast<Harness*>(hp);
        const std::string p(prefix);
        const size_t n = h->events.size();
        std::vector<uint32_t> u[5];
        std::vector<float> f[5];
        for (auto& v : u) v.resize(n);
        for (auto& v : f) v.resize(n);
        for (size_t i = 0; i < n; i++)
        {
            const auto& e = h->events[i];
            u[0][i] = e.self; u[1][i] = e.other; u[2][i] = e.selfBody; u[3][i] = e.otherBody; u[4][i] = e.callback;
            f[0][i] = e.px; f[1][i] = e.py; f[2][i] = e.nx; f[3][i] = e.ny; f[4][i] = e.impulse;
        }
        const char* un[5] = {"ev.self", "ev.other", "ev.selfBody", "ev.otherBody", "ev.callback"};
        const char* fn[5] = {"ev.px", "ev.py", "ev.nx", "ev.ny", "ev.impulse"};
        for (int k = 0; k < 5; k++) { h->putv(p + un[k], u[k]); h->putv(p + fn[k], f[k]); }
        h->events.clear();
    }

    // Constraints (ConstraintAPI::createSpring / createRevoluteJoint / createMotor, SimulationAPIs/ConstraintAPI.h:
    // 32-36) between bodies given by handle slot; returns the constraint's handle slot or -1 (stale body).
    // kind 0 spring (p: anchorA xy, anchorB xy, rest length, stiffness, damping), 1 revolute joint (anchors,
    // stiffness, damping), 2 prismatic and 3 slider joint (anchors, local axis xy, stiffness, damping, lower and
    // upper limit, limit enabled), 4 motor (body A only; p: target speed, max torque).
    int64_t agref_create_joint(void* hp, int32_t kind, uint32_t slotA, uint32_t slotB, const float* p)
    {
        auto* h = static_cast<Harness*>(hp);
        auto& o = h->sim.objectManager;
        const Handle a = bodyHandleOfSlot(h, slotA), b = bodyHandleOfSlot(h, slotB);
        std::optional<Handle> r;
        switch (kind)
        {
        case 0: r = o.createSpring({a, b, Vec2(p[0], p[1]), Vec2(p[2], p[3]), p[4], p[5], p[6]}); break;
        case 1: r = o.createRevoluteJoint({a, b, Vec2(p[0], p[1]), Vec2(p[2], p[3]), p[4], p[5]}); break;
        case 2: {
            PrismaticJointConstraintSystem::CreateParams q{a, b, Vec2(p[0], p[1]), Vec2(p[2], p[3]), Vec2(p[4], p[5]),
                                                           p[6], p[7]};
            q.lowerLimit = p[8]; q.upperLimit = p[9]; q.enableLimit = p[10] != 0.0f;
            r = o.createPrismaticJoint(q);
            break;
        }
        case 3: {
            SliderJointConstraintSystem::CreateParams q{a, b, Vec2(p[0], p[1]), Vec2(p[2], p[3]), Vec2(p[4], p[5]),
                                                        p[6], p[7]};
            q.lowerLimit = p[8]; q.upperLimit = p[9]; q.enableLimit = p[10] != 0.0f;
            r = o.createSliderJoint(q);
            break;
        }
        case 4: r = o.createMotor({a, p[0], p[1]}); break;
        default: break;
        }
        return r ? int64_t(r->slot) : -1;
    }
    // A constraint system's dense order as handles (slot, generation) and its group starts (Inactive, Sleeping,
    // Active, end): ConstraintAPI::get*Handle over every dense index. Returns the count.
    uint32_t agref_joint_order(void* hp, int32_t kind, uint32_t* slot, uint32_t* gen, uint32_t* starts, uint32_t cap)
    {
        auto* h = static_cast<Harness*>(hp);
        IConstraintSystem* sys = h->sim.constraintSystems[size_t(kind)];
        const uint32_t n = uint32_t(sys->getCount());
        for (uint32_t i = 0; i < n && i < cap; i++)
        {
            Handle hd{};
            switch (kind)
            {
            case 0: hd = h->sim.springConstraintSystem.handleAt(i); break;
            case 1: hd = h->sim.jointConstraintSystem.handleAt(i); break;
            case 2: hd = h->sim.prismaticJointConstraintSystem.handleAt(i); break;
            case 3: hd = h->sim.sliderJointConstraintSystem.handleAt(i); break;
            default: hd = h->sim.motorConstraintSystem.handleAt(i); break;
            }
            slot[i] = hd.slot;
            gen[i] = hd.generation;
        }
        for (int g = 0; g < 4; g++) starts[g] = sys->groupStarts[g];
        return n;
    }
    // Deferred constraint destroy (ConstraintAPI::destroy*, applied at the next flush).
    void agref_destroy_joint(void* hp, int32_t kind, uint32_t slot, uint32_t gen)
    {
        static_cast<Harness*>(hp)->sim.objectManager.destroyConstraint(ConstraintType(kind), Handle{slot, gen});
    }

    // The motors' accumulated impulses and body handle slots in dense order (MotorSoA).
    uint32_t agref_motor_impulses(void* hp, float* impulse, uint32_t* bodySlot, uint32_t cap)
    {
        auto* h = static_cast<Harness*>(hp);
        auto& sys = h->sim.motorConstraintSystem;
        const auto view = sys.getViewer();
        const uint32_t n = uint32_t(sys.getCount());
        for (uint32_t i = 0; i < n && i < cap; i++)
        {
            impulse[i] = view.accumulatedImpulse[i];
            bodySlot[i] = h->sim.objectManager.bodies.handleAt(view.bodyIndex[i]).slot;
        }
        return n;
    }

    // Dense body index of a handle slot (UINT32_MAX when destroyed).
    uint32_t agref_body_index(void* hp, uint32_t slot)
    {
        auto* h = static_cast<Harness*>(hp);
        return h->sim.objectManager.bodies.indexOf(bodyHandleOfSlot(h, slot));
    }

    int64_t agref_add_collider(void* hp, uint32_t slot, int32_t shape, float lx, float ly, float lrot, uint32_t mat,
                               float p0, float p1, const float* xy, uint32_t n)
    {
        auto* h = static_cast<Harness*>(hp);
        auto& o = h->sim.objects();
        const Handle body = bodyHandleOfSlot(h, slot);
        std::optional<ObjectDenseIndex> c;
        switch (shape)
        {
        case 0: c = o.createCircleCollider({.bodyHandle = body, .localOffset = Vec2(lx, ly), .localRotation = lrot,
                                            .materialIndex = mat, .radius = p0}); break;
        case 1: c = o.createBoxCollider({.bodyHandle = body, .localOffset = Vec2(lx, ly), .localRotation = lrot,
                                         .materialIndex = mat, .size = Vec2(p0, p1)}); break;
        case 2: {
            std::vector<Vec2> v(n);
            for (uint32_t i = 0; i < n; i++) v[i] = Vec2(xy[2 * i], xy[2 * i + 1]);
            PolygonColliderCreateParams p;
            p.bodyHandle = body; p.localOffset = Vec2(lx, ly); p.localRotation = lrot; p.materialIndex = mat;
            p.localVertices = v.data(); p.verticesCount = n;
            auto r = o.createPolygonCollider(p);
            if (r) c = r->firstColliderIndex;
            break;
        }
        case 3: c = o.createCapsuleCollider({.bodyHandle = body, .localOffset = Vec2(lx, ly), .localRotation = lrot,
                                             .materialIndex = mat, .length = p0, .radius = p1}); break;
        default: break;
        }
        return c ? int64_t(*c) : -1;
    }

    // Steps through the reference's public entry point, Simulation::update (Simulation.cpp:32-74). With
    // updateInterval == dt every call takes exactly one fixed step (FixedClock.h:35-63).
    void agref_update(void* hp, int32_t steps)
    {
        auto* h = static_cast<Harness*>(hp);
        useBackend(h);
        for (int32_t i = 0; i < steps; i++) h->sim.update(h->dt);
    }

    // Wall-clock seconds for 'steps' updates (the CPU baseline timer).
    double agref_timed_update(void* hp, int32_t steps)
    {
        auto* h = static_cast<Harness*>(hp);
        useBackend(h);
        const auto t0 = std::chrono::steady_clock::now();
        for (int32_t i = 0; i < steps; i++) h->sim.update(h->dt);
        const auto t1 = std::chrono::steady_clock::now();
        return std::chrono::duration<double>(t1 - t0).count();
    }

    // Wall-clock seconds of the collision detection part of one step on the current state, as collisionStep runs
    // it (Simulation.cpp:410-421): spatial data (poses, AABBs, trees), broad phase, narrow phase. Nothing is
    // integrated or solved. Reports the pair and manifold counts.
    double agref_timed_collide(void* hp, uint64_t* out_pairs, uint64_t* out_manifolds)
    {
        auto* h = static_cast<Harness*>(hp);
        useBackend(h);
        Simulation& s = h->sim;
        s.flushCommands();
        s.setDataViewers();
        const auto t0 = std::chrono::steady_clock::now();
        if (s.objectManager.spatialDirty) s.rebuildSpatialData();
        else s.updateDynamicSpatialData();
        std::span<const ObjectPair> broad{};
        std::span<BodyCollisionData> narrow{};
        if (s.objectManager.colliders.getCount() > 1) {
            broad = s.broadPhaseCollisionDetector.findCollisions(ExecutionPolicy::ForceSingleThreaded);
            if (!broad.empty()) narrow = s.narrowPhaseCollisionDetector.findCollisions(broad);
        }
        const auto t1 = std::chrono::steady_clock::now();
        if (out_pairs) *out_pairs = broad.size();
        if (out_manifolds) *out_manifolds = narrow.size();
        return std::chrono::duration<double>(t1 - t0).count();
    }

    uint32_t agref_body_count(void* hp) { return uint32_t(static_cast<Harness*>(hp)->sim.objectManager.bodies.getCount()); }
    uint32_t agref_collider_count(void* hp) { return uint32_t(static_cast<Harness*>(hp)->sim.objectManager.colliders.getCount()); }
    uint32_t agref_manifold_count(void* hp) { return uint32_t(static_cast<Harness*>(hp)->sim.getBodyCollisionData().size()); }

    void agref_dump_state(void* hp, const char* prefix)
    {
        auto* h = static_cast<Harness*>(hp);
        const std::string p(prefix);
        dumpBodies(h, p);
        dumpColliders(h, p);
        dumpManifolds(h, p + "man.", h->sim.getBodyCollisionData());
        dumpIslandStore(h, p + "isle.");
    }

    // Overwrites one float field of every body (used to drive the integration/wrap/cos-sin phases with chosen
    // inputs). Returns 0 on success, -1 for an unknown field.
    int32_t agref_set_body_field(void* hp, const char* field, const float* data)
    {
        BodySoA& b = static_cast<Harness*>(hp)->sim.objectManager.bodies;
        const std::string f(field);
        CacheLineAlignedVector<Real>* dst = nullptr;
        if (f == "velocityX") dst = &b.velocityX;
        else if (f == "velocityY") dst = &b.velocityY;
        else if (f == "rotation") dst = &b.rotation;
        else if (f == "angularVelocity") dst = &b.angularVelocity;
        else if (f == "comX") dst = &b.comX;
        else if (f == "comY") dst = &b.comY;
        if (!dst) return -1;
        std::memcpy(dst->data(), data, dst->size() * sizeof(Real));
        return 0;
    }

    // One fixed step with taps between the phases. Mirrors the member-function sequence of Simulation::update
    // (flushCommands, preUpdate, physicsStep, postUpdate; Simulation.cpp:32-74, 255-351, 410-451) and records:
    //   pre.*  state entering the step          int.*  after integration, wrap, rotation cos/sin
    //   sp.*   collider poses + AABBs           dyn.*  dynamic tree (Morton-sorted collider indices and keys)
    //   bp.pairs  broad-phase collider pairs    np.*   narrow-phase manifolds incl. warm-start impulses
    //   sv.*   after the contact solver         is.*   island ids        post.*  state after the step
    void agref_phase_step(void* hp)
    {
        auto* h = static_cast<Harness*>(hp);
        useBackend(h);
        Simulation& s = h->sim;
        const Real dt = h->dt;

        s.flushCommands();
        s.clock.setSettings(s.simulationSettings.clockSettings);
        s.clock.advance(dt);
        s.preUpdate();

        dumpBodies(h, "pre.");
        dumpColliders(h, "pre.");
        dumpManifolds(h, "pre.man.", s.narrowPhaseCollisionDetector.getBodyCollisionData());
        dumpIslandStore(h, "pre.isle.");

        s.simulationRunTimer += dt;
        s.bodyCollisionSolver.resetCollisionData();
        s.bodyCollisionSolver.setCollisionEventRecording(false);
        if (s.objectManager.bodies.getCount() == 0) return;
        s.wakeHeldBodies();
        s.setDataViewers();

        const bool ccd = s.simulationSettings.continuousCollisionEnabled;
        if (ccd) {
            s.continuousCollisionDetector.settings = s.simulationSettings.ccdSettings;
            s.continuousCollisionDetector.snapshotPoses(s.objectManager.bodies, s.objectManager.colliders);
        }
        s.integrateAndApplyConstraints(dt);
        const IndexRange dynamicRange = s.objectManager.bodies.range(BodyGroup::Dynamic);
        wrapBodyRotations(s.objectManager.bodies, dynamicRange);
        Integrator::computeRotationCosSin(s.objectManager.bodies, dynamicRange);
        dumpBodies(h, "int.");

        const bool wasDirty = s.objectManager.spatialDirty;
        if (s.objectManager.spatialDirty) s.rebuildSpatialData();
        else s.updateDynamicSpatialData();
        uint32_t dirtyFlag = wasDirty ? 1u : 0u;
        h->put("sp.spatialDirty", &dirtyFlag, 1);
        dumpColliders(h, "sp.");
        // Continuous collision as physicsStep runs it (Simulation.cpp:299-316): tap "ccd." after the move-back.
        if (ccd) {
            const auto* staticTreePtr = s.broadPhaseCollisionDetector.getTree(BroadPhaseInternal::BvhTreeType::Static);
            uint32_t hit = 0;
            if (staticTreePtr) {
                hit = s.continuousCollisionDetector.resolve(s.objectManager.bodies, s.objectManager.colliders,
                                                            s.objectManager.circles, s.objectManager.boxes,
                                                            s.objectManager.polygons, s.objectManager.capsules,
                                                            *staticTreePtr) ? 1u : 0u;
                if (hit) {
                    s.buildColliderAABBs(false);
                    s.broadPhaseCollisionDetector.refitTrees(BroadPhaseInternal::BvhTreeTypeFlag::Dynamic);
                }
            }
            h->put("ccd.hit", &hit, 1);
            dumpBodies(h, "ccd.");
            dumpColliders(h, "ccd.");
        }
        dumpTree(h, "dyn.", BroadPhaseInternal::BvhTreeType::Dynamic);
        dumpTree(h, "static.", BroadPhaseInternal::BvhTreeType::Static);
        dumpTree(h, "sleep.", BroadPhaseInternal::BvhTreeType::Sleeping);

        s.islandBodyCollisionEdges = {};
        std::span<const ObjectPair> broad{};
        std::span<BodyCollisionData> narrow{};
        if (s.objectManager.colliders.getCount() > 1)
        {
            broad = s.broadPhaseCollisionDetector.findCollisions(ExecutionPolicy::ForceSingleThreaded);
            h->put("bp.pairs", reinterpret_cast<const uint32_t*>(broad.data()), 2 * broad.size());
            if (broad.empty())
            {
                s.narrowPhaseCollisionDetector.resetCollisionData();
            }
            else
            {
                narrow = s.narrowPhaseCollisionDetector.findCollisions(broad);
                dumpManifolds(h, "np.", narrow);
                if (narrow.empty())
                {
                    s.narrowPhaseCollisionDetector.rebuildContactCache();
                }
                else
                {
                    s.objectManager.wakeIslandsOfContacts(narrow);
                    s.wakeSleepingContactData();
                    narrow = s.narrowPhaseCollisionDetector.getBodyCollisionData();
                    s.islandBodyCollisionEdges = s.bodyCollisionSolver.fillCollidingBodyPairs(narrow);
                    dumpBodies(h, "svin.");
                    dumpColliders(h, "svin.");
                    dumpManifolds(h, "svin.man.", narrow);
                    s.bodyCollisionSolver.solveCollisions(
                        narrow,
                        s.simulationSettings.collisionVelocitySolvingIterations,
                        s.simulationSettings.collisionPositionSolvingIterations);
                    dumpBodies(h, "sv.");
                    dumpManifolds(h, "sv.man.", narrow);
                    s.narrowPhaseCollisionDetector.rebuildContactCache();
                    s.dispatchCollisionEvents();
                }
            }
        }
        else
        {
            s.narrowPhaseCollisionDetector.resetCollisionData();
        }

        s.islandManager.reset(s.objectManager.bodies);
        s.islandManager.step(s.islandBodyCollisionEdges);
        for (auto* cs : s.constraintSystems) s.islandManager.step(cs->getActiveEdges());
        s.islandManager.finalize(s.objectManager.bodies);
        h->putv("is.islandId", s.objectManager.bodies.islandId);

        s.flushCommands();
        s.updateSleeping(float(dt));
        s.sleepContactData();
        s.postUpdate();

        dumpBodies(h, "post.");
        dumpColliders(h, "post.");
        dumpManifolds(h, "post.man.", s.getBodyCollisionData());
        dumpIslandStore(h, "post.isle.");
    }

    uint64_t agref_blob_size(void* hp, const char* name)
    {
        auto* h = static_cast<Harness*>(hp);
        auto it = h->blobs.find(name);
        return it == h->blobs.end() ? ~0ull : uint64_t(it->second.size());
    }

    int32_t agref_blob_copy(void* hp, const char* name, void* dst)
    {
        auto* h = static_cast<Harness*>(hp);
        auto it = h->blobs.find(name);
        if (it == h->blobs.end()) return -1;
        if (!it->second.empty()) std::memcpy(dst, it->second.data(), it->second.size());
        return 0;
    }

    // Newline-separated blob names (for discovery); returns the byte length needed including the terminator.
    uint64_t agref_blob_names(void* hp, char* dst, uint64_t cap)
    {
        auto* h = static_cast<Harness*>(hp);
        std::string all;
        for (auto& kv : h->blobs) { all += kv.first; all += '\n'; }
        if (dst && cap > all.size()) std::memcpy(dst, all.c_str(), all.size() + 1);
        return uint64_t(all.size() + 1);
    }

    void agref_clear_blobs(void* hp) { static_cast<Harness*>(hp)->blobs.clear(); }

    // Colliders a shape query finds through the reference's own trees (BroadPhaseCollisionDetector::
    // queryCollidersInShape, BroadPhaseCollisionDetector.h:189-203, with AABBQuery / CircleQuery, QueryShapes.h):
    // shape 0 = AABB {minX, minY, maxX, maxY}, 1 = circle {x, y, radius}; 'trees' the BvhTreeTypeFlag bits. Returns
    // the count and writes at most 'cap' dense collider indices, in the reference's traversal order.
    int64_t agref_query_shape(void* hp, int32_t shape, const float* p, uint32_t trees, uint32_t* out, uint64_t cap)
    {
        auto* h = static_cast<Harness*>(hp);
        std::vector<ObjectDenseIndex> found;
        const BroadPhaseCollisionDetector& bp = h->sim.getBroadPhaseCollisionDetector();
        const auto flags = static_cast<BroadPhaseInternal::BvhTreeTypeFlag>(trees);
        if (shape == 0) {
            AABB box;
            box.minX = p[0]; box.minY = p[1]; box.maxX = p[2]; box.maxY = p[3];
            bp.queryCollidersInShape(BroadPhaseInternal::AABBQuery(box), flags, found);
        } else {
            bp.queryCollidersInShape(BroadPhaseInternal::CircleQuery(Vec2{p[0], p[1]}, p[2]), flags, found);
        }
        for (size_t i = 0; i < found.size() && i < cap; i++) out[i] = uint32_t(found[i]);
        return int64_t(found.size());
    }

    // Colliders a circle touches: the circle query's colliders (as above) passed to
    // NarrowPhaseCollisionDetector::findCollisionsInCircle (NarrowPhaseCollisionDetector.cpp:153-270). Returns the
    // count; writes at most 'cap' (collider, signed distance) results in the reference's order.
    int64_t agref_circle_contacts(void* hp, float x, float y, float r, uint32_t trees, uint32_t* outIdx, float* outSdf,
                                  uint64_t cap)
    {
        auto* h = static_cast<Harness*>(hp);
        std::vector<ObjectDenseIndex> found;
        h->sim.getBroadPhaseCollisionDetector().queryCollidersInShape(
            BroadPhaseInternal::CircleQuery(Vec2{x, y}, r), static_cast<BroadPhaseInternal::BvhTreeTypeFlag>(trees),
            found);
        std::vector<std::pair<ObjectDenseIndex, Real>> hits;
        h->sim.getNarrowPhaseCollisionDetector().findCollisionsInCircle(found, Vec2{x, y}, r, hits);
        for (size_t i = 0; i < hits.size() && i < cap; i++) {
            outIdx[i] = uint32_t(hits[i].first);
            outSdf[i] = float(hits[i].second);
        }
        return int64_t(hits.size());
    }

    // The reference's batched rotation cos/sin over an array (FastCosSin.cpp:26-109), SIMD body and scalar tail.
    void agref_fastcossin(const float* in, float* outCos, float* outSin, uint64_t n)
    {
        FastCosSin::order5Array(in, outCos, outSin, size_t(n));
    }
}
