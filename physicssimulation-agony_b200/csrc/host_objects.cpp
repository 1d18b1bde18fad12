// Host-side object bookkeeping (see host_objects.hpp). Compiled with -ffp-contract=off: the creation arithmetic
// must round like the reference's parity build.
#include "host_objects.hpp"

#include <algorithm>
#include <cfloat>
#include <limits>

namespace ag2d {

bool polygon_inertia(float mass, const std::vector<float>& xy, float& inertia, float& cx, float& cy)
{
    const size_t n = xy.size() / 2;
    if (n < 3) return false;
    float signedArea = 0, sx = 0, sy = 0, xx = 0, yy = 0;
    for (size_t i = 0; i < n; i++) {
        const size_t j = (i + 1 == n) ? 0 : i + 1;
        const float p0x = xy[2 * i], p0y = xy[2 * i + 1], p1x = xy[2 * j], p1y = xy[2 * j + 1];
        const float cross = p0x * p1y - p1x * p0y;
        signedArea += cross;
        sx += (p0x + p1x) * cross;
        sy += (p0y + p1y) * cross;
        xx += (p0y * p0y + p0y * p1y + p1y * p1y) * cross;
        yy += (p0x * p0x + p0x * p1x + p1x * p1x) * cross;
    }
    signedArea *= 0.5f;
    if (signedArea < std::numeric_limits<float>::epsilon()) return false;
    const float invSixArea = 1.0f / (6.0f * signedArea);
    cx = sx * invSixArea;
    cy = sy * invSixArea;
    inertia = (mass / signedArea) * ((xx + yy) / 12.0f) - mass * (cx * cx + cy * cy);
    return true;
}

namespace {

// PhysicsGeometry::filterDuplicateVertices (PhysicsGeometry.cpp:314-347), eps 1e-5.
std::vector<float> filter_duplicates(const float* xy, uint32_t n)
{
    const float epsSq = 1e-5f * 1e-5f;
    auto close = [epsSq](float ax, float ay, float bx, float by) {
        const float dx = ax - bx, dy = ay - by;
        return dx * dx + dy * dy <= epsSq;
    };
    std::vector<float> out;
    for (uint32_t i = 0; i < n; i++) {
        const size_t m = out.size() / 2;
        if (m == 0 || !close(out[2 * m - 2], out[2 * m - 1], xy[2 * i], xy[2 * i + 1])) {
            out.push_back(xy[2 * i]);
            out.push_back(xy[2 * i + 1]);
        }
    }
    while (out.size() / 2 > 1 && close(out[out.size() - 2], out[out.size() - 1], out[0], out[1])) {
        out.pop_back();
        out.pop_back();
    }
    return out;
}

}  // namespace

// PhysicsGeometry::preparePolygonOutline (PhysicsGeometry.cpp:175-212): dedupe, strip straight vertices, make CCW,
// reject degenerate and non-simple outlines.
bool prepare_outline_any(const float* xy, uint32_t n, std::vector<float>& out, std::string& err)
{
    out = filter_duplicates(xy, n);
    bool removed = true;
    while (removed && out.size() / 2 >= 3) {
        removed = false;
        const size_t m = out.size() / 2;
        std::vector<float> kept;
        for (size_t i = 0; i < m; i++) {
            const size_t p = (i + m - 1) % m, q = (i + 1) % m;
            const float e1x = out[2 * i] - out[2 * p], e1y = out[2 * i + 1] - out[2 * p + 1];
            const float e2x = out[2 * q] - out[2 * i], e2y = out[2 * q + 1] - out[2 * i + 1];
            const float len1 = std::sqrt(e1x * e1x + e1y * e1y), len2 = std::sqrt(e2x * e2x + e2y * e2y);
            const bool straight = (e1x * e2x + e1y * e2y) > 0.0f &&
                                  std::abs(e1x * e2y - e1y * e2x) <= 1e-6f * len1 * len2;
            if (straight) removed = true;
            else { kept.push_back(out[2 * i]); kept.push_back(out[2 * i + 1]); }
        }
        out.swap(kept);
    }
    const size_t m = out.size() / 2;
    if (m < 3) { err = "polygon outline is degenerate"; return false; }
    float area2 = 0;
    for (size_t i = 0; i < m; i++) {
        const size_t j = (i + 1) % m;
        area2 += out[2 * i] * out[2 * j + 1] - out[2 * j] * out[2 * i + 1];
    }
    if (area2 < 0.0f) {
        std::vector<float> rev(out.size());
        for (size_t i = 0; i < m; i++) { rev[2 * i] = out[2 * (m - 1 - i)]; rev[2 * i + 1] = out[2 * (m - 1 - i) + 1]; }
        out.swap(rev);
    }
    if (std::abs(area2) * 0.5f <= std::numeric_limits<float>::epsilon()) { err = "polygon outline is degenerate"; return false; }
    if (!outline_is_simple(out)) { err = "polygon outline is self-intersecting"; return false; }
    return true;
}

bool prepare_outline(const float* xy, uint32_t n, std::vector<float>& out, std::string& err)
{
    if (!prepare_outline_any(xy, n, out, err)) return false;
    if (out.size() / 2 > 16) { err = "polygon has more than 16 vertices (MAX_POLYGON_VERTEX_COUNT)"; return false; }
    if (!outline_is_convex(out)) { err = "polygon is not convex"; return false; }
    return true;
}

// PolygonGeometry::computeNormals (SoA/Shapes/PolygonSoA.cpp:14-30).
std::vector<float> polygon_normals(const std::vector<float>& v)
{
    const size_t n = v.size() / 2;
    std::vector<float> nrm(v.size());
    for (size_t i = 0; i < n; i++) {
        const size_t j = (i + 1 == n) ? 0 : i + 1;
        const float ex = v[2 * j] - v[2 * i], ey = v[2 * j + 1] - v[2 * i + 1];
        float nx = ey, ny = -ex;
        const float lenSq = nx * nx + ny * ny;
        if (lenSq >= 1e-8f) {
            const float inv = 1.0f / std::sqrt(lenSq);
            nx = nx * inv;
            ny = ny * inv;
        } else {
            nx = 0.0f;
            ny = 0.0f;
        }
        nrm[2 * i] = nx;
        nrm[2 * i + 1] = ny;
    }
    return nrm;
}

uint32_t HostObjects::appendBody(float px, float py, float vx, float vy, float rot, float w, float mass,
                                 float invMass, float inertia, float invInertia, float lcomX, float lcomY)
{
    // ObjectManager::appendBody (ObjectManager.cpp:1269-1286) and BodySoA::append (SoA/BodySoA.cpp:6-40).
    const float cosR = std::cos(rot), sinR = std::sin(rot);
    HBody b;
    b.comX = px + (cosR * lcomX - sinR * lcomY);
    b.comY = py + (sinR * lcomX + cosR * lcomY);
    b.vx = vx; b.vy = vy; b.rot = rot; b.w = w;
    b.mass = mass; b.invMass = invMass; b.inertia = inertia; b.invInertia = invInertia;
    b.lcomX = lcomX; b.lcomY = lcomY;
    b.cos = std::cos(rot);
    b.sin = std::sin(rot);
    // Handle table push (HandleTable.h:29-45).
    b.handleSlot = uint32_t(slotIndex.size());
    slotIndex.push_back(uint32_t(bodies.size()));
    slotGeneration.push_back(0);
    bodies.push_back(std::move(b));   // the new body sits in the unused range [starts[3], count)
    return moveBodyDown(uint32_t(bodies.size() - 1), invMass == 0.0f ? 0u : 2u);
}

// ---- constraint systems ----

void JointSystem::swap(uint32_t a, uint32_t b)
{
    if (a == b) return;
    std::swap(joints[a], joints[b]);
    slotIndex[joints[a].handleSlot] = a;
    slotIndex[joints[b].handleSlot] = b;
}

uint32_t JointSystem::moveToGroup(uint32_t index, uint32_t target)
{
    uint32_t g = groupOf(index);
    while (g != target) {
        if (g < target) {   // to the group's last slot, then across the boundary above it
            const uint32_t last = starts[g + 1] - 1;
            swap(index, last);
            index = last;
            starts[g + 1]--;
            g++;
        } else {            // to the group's first slot, then across the boundary below it
            const uint32_t first = starts[g];
            swap(index, first);
            index = first;
            starts[g]++;
            g--;
        }
    }
    return index;
}

uint32_t JointSystem::create(const HJoint& j, uint32_t group)
{
    uint32_t slot;
    if (freeHead != NO_BODY) {
        slot = freeHead;
        freeHead = slotIndex[slot];
    } else {
        slot = uint32_t(slotIndex.size());
        slotIndex.push_back(0);
        slotGeneration.push_back(0);
    }
    joints.push_back(j);
    joints.back().handleSlot = slot;
    const uint32_t index = uint32_t(joints.size() - 1);
    slotIndex[slot] = index;   // appended in the unused range, then moved down to its group
    return moveToGroup(index, group);
}

void JointSystem::destroy(uint32_t index)
{
    if (index >= joints.size()) return;
    index = moveToGroup(index, JGROUP_UNUSED);
    swap(index, uint32_t(joints.size() - 1));
    const uint32_t slot = joints.back().handleSlot;
    joints.pop_back();
    slotGeneration[slot]++;
    slotIndex[slot] = freeHead;
    freeHead = slot;
}

void HostObjects::swapBodies(uint32_t a, uint32_t b)
{
    if (a == b) return;
    for (JointSystem& js : jointSystems)
        for (HJoint& j : js.joints) {
            if (j.bodyA == a) j.bodyA = b; else if (j.bodyA == b) j.bodyA = a;
            if (j.bodyB == a) j.bodyB = b; else if (j.bodyB == b) j.bodyB = a;
        }
    std::swap(bodies[a], bodies[b]);
    for (uint32_t c : bodies[a].colliders) colliders[c].body = a;
    for (uint32_t c : bodies[b].colliders) colliders[c].body = b;
    slotIndex[bodies[a].handleSlot] = a;
    slotIndex[bodies[b].handleSlot] = b;
}

void HostObjects::swapColliders(uint32_t a, uint32_t b)
{
    if (a == b) return;
    std::swap(colliders[a], colliders[b]);
    for (uint32_t& c : bodies[colliders[a].body].colliders) if (c == b) { c = a; break; }
    for (uint32_t& c : bodies[colliders[b].body].colliders) if (c == a) { c = b; break; }
}

// moveBodyToGroup for a freshly appended body (ObjectManager.cpp:1232-1267): moving down a group swaps with that
// group's first body and advances the group's start.
uint32_t HostObjects::moveBodyDown(uint32_t index, uint32_t target)
{
    uint32_t g = 3;
    while (g != target) {
        const uint32_t first = g == 3 ? bodyGroups.starts[3] : bodyGroups.starts[g];
        swapBodies(index, first);
        index = first;
        bodyGroups.starts[g]++;
        g--;
    }
    return index;
}

uint32_t HostObjects::moveColliderDown(uint32_t index, uint32_t target)
{
    uint32_t g = 3;
    while (g != target) {
        const uint32_t first = colGroups.starts[g];
        swapColliders(index, first);
        index = first;
        colGroups.starts[g]++;
        g--;
    }
    return index;
}

uint32_t HostObjects::appendCollider(uint32_t body, float locX, float locY, float localRot, uint32_t material,
                                     uint32_t type, uint32_t shape, float minExt, float maxExt)
{
    // ObjectManager::createColliderInternal + placeNewCollider (ObjectManager.cpp:522-533, 1103-1108); comOffset =
    // localOffset - body local centre of mass (refreshComOffset, :17-22).
    // The local rotation is stored wrapped into [0, 2pi) (ColliderSoA::append, SoA/ColliderSoA.cpp:25-27); the
    // polygon recentring before this call used the rotation as given.
    const float twoPi = 6.28318548f;   // 2 * float(pi)
    float wrapped = std::fmod(localRot, twoPi);
    if (wrapped < 0.0f) wrapped += twoPi;
    HCollider c;
    c.body = body; c.locX = locX; c.locY = locY; c.localRot = wrapped; c.material = material;
    c.type = type; c.shape = shape; c.minExtent = minExt; c.maxExtent = maxExt;
    c.comOffX = locX - bodies[body].lcomX;
    c.comOffY = locY - bodies[body].lcomY;
    colliders.push_back(c);
    const uint32_t idx = uint32_t(colliders.size() - 1);
    bodies[body].colliders.push_back(idx);
    const float reach = std::sqrt(c.comOffX * c.comOffX + c.comOffY * c.comOffY) + c.maxExtent;
    bodies[body].boundRadius = std::fmax(bodies[body].boundRadius, reach);
    return moveColliderDown(idx, bodyGroups.groupOf(body));
}

bool HostObjects::addCircle(const float* d, uint32_t material, float radius, uint64_t& handle, std::string& err)
{
    if (!(radius >= 0.0f)) { err = "radius must be >= 0"; return false; }
    if (material >= materialCount()) material = 0;
    // ObjectManager::createCircle (ObjectManager.cpp:233-257); calculateCircleInertia (PhysicsGeometry.cpp:116-121).
    const float mass = std::fmax(0.0f, d[6]);
    const float r = std::fmax(0.0f, radius);
    const float inertia = (0.5f * (r * r) + 0.0f) * mass;
    const float invMass = mass == 0.0f ? 0.0f : 1.0f / mass;
    const float invInertia = inertia == 0.0f ? 0.0f : 1.0f / inertia;
    const uint32_t b = appendBody(d[0], d[1], d[3], d[4], d[2], d[5], mass, invMass, inertia, invInertia, 0.0f, 0.0f);
    const uint32_t slot = bodies[b].handleSlot;
    circleRadius.push_back(r);
    appendCollider(b, 0.0f, 0.0f, 0.0f, material, 0u, uint32_t(circleRadius.size() - 1), r, r);
    handle = (uint64_t(slotGeneration[slot]) << 32) | slot;
    return true;
}

bool HostObjects::addBox(const float* d, uint32_t material, float width, float height, uint64_t& handle,
                         std::string& err)
{
    if (!(width >= 0.0f && height >= 0.0f)) { err = "box size must be >= 0"; return false; }
    if (material >= materialCount()) material = 0;
    // ObjectManager::createBox (ObjectManager.cpp:259-284); calculateBoxInertia (PhysicsGeometry.cpp:123-128).
    const float mass = std::fmax(0.0f, d[6]);
    const float w = std::fmax(0.0f, width), h = std::fmax(0.0f, height);
    const float div = float(1.0 / 12.0);
    const float inertia = mass * (div * (w * w + h * h) + 0.0f);
    const float invMass = mass == 0.0f ? 0.0f : 1.0f / mass;
    const float invInertia = inertia == 0.0f ? 0.0f : 1.0f / inertia;
    const uint32_t b = appendBody(d[0], d[1], d[3], d[4], d[2], d[5], mass, invMass, inertia, invInertia, 0.0f, 0.0f);
    const uint32_t slot = bodies[b].handleSlot;
    const float hw = w * 0.5f, hh = h * 0.5f;
    boxHalfW.push_back(hw);
    boxHalfH.push_back(hh);
    appendCollider(b, 0.0f, 0.0f, 0.0f, material, 1u, uint32_t(boxHalfW.size() - 1), std::fmin(hw, hh),
                   std::fmax(hw, hh));
    handle = (uint64_t(slotGeneration[slot]) << 32) | slot;
    return true;
}

bool HostObjects::addPolygon(const float* d, uint32_t material, const float* xy, uint32_t n, uint64_t& handle,
                             std::string& err)
{
    if (!xy || n < 3) { err = "polygon needs at least 3 vertices"; return false; }
    if (material >= materialCount()) material = 0;
    // ObjectManager::createPolygon (ObjectManager.cpp:286-349) via PhysicsGeometry::buildPolygon (:361-400).
    const float mass = std::fmax(0.0f, d[6]);
    std::vector<float> outline;
    if (!prepare_outline_any(xy, n, outline, err)) return false;
    float inertia = 0, tcx = 0, tcy = 0;
    if (!polygon_inertia(mass, outline, inertia, tcx, tcy)) { err = "polygon outline is degenerate"; return false; }
    const float needX = tcx - tcx, needY = tcy - tcy;   // requested pivot defaults to the true centre of mass
    for (size_t i = 0; i < outline.size() / 2; i++) { outline[2 * i] -= tcx; outline[2 * i + 1] -= tcy; }
    inertia = inertia + mass * (needX * needX + needY * needY);
    // Convex pieces of the centred outline (decomposeConcave + limitConvexPieceVertexCount), one collider each.
    std::vector<std::vector<float>> pieces = decompose_outline(outline, 16);
    if (pieces.empty()) { err = "decomposition produced no pieces"; return false; }
    const float cosR = std::cos(d[2]), sinR = std::sin(d[2]);
    const float ox = d[0] + (cosR * tcx - sinR * tcy);
    const float oy = d[1] + (sinR * tcx + cosR * tcy);
    const float invMass = mass == 0.0f ? 0.0f : 1.0f / mass;
    const float invInertia = inertia == 0.0f ? 0.0f : 1.0f / inertia;
    const uint32_t b = appendBody(ox, oy, d[3], d[4], d[2], d[5], mass, invMass, inertia, invInertia, needX, needY);
    const uint32_t slot = bodies[b].handleSlot;
    for (const std::vector<float>& piece : pieces) appendPolygonPiece(b, 0.0f, 0.0f, 0.0f, material, piece);
    handle = (uint64_t(slotGeneration[slot]) << 32) | slot;
    return true;
}

// createConvexPolygonColliderInternal (ObjectManager.cpp:535-562): recentre the piece on its own centroid and move
// the shift into the local offset; extents are the in-radius and out-radius about the new origin.
uint32_t HostObjects::appendPolygonPiece(uint32_t b, float offX, float offY, float localRot, uint32_t material,
                                         std::vector<float> outline)
{
    float unused = 0, pcx = 0, pcy = 0;
    polygon_inertia(1.0f, outline, unused, pcx, pcy);
    for (size_t i = 0; i < outline.size() / 2; i++) { outline[2 * i] -= pcx; outline[2 * i + 1] -= pcy; }
    const float cosL = std::cos(localRot), sinL = std::sin(localRot);
    const float locX = offX + (cosL * pcx - sinL * pcy);
    const float locY = offY + (sinL * pcx + cosL * pcy);
    HPolygon poly;
    poly.verts = outline;
    poly.normals = polygon_normals(outline);
    float inR = FLT_MAX, outR2 = 0.0f;
    for (size_t i = 0; i < outline.size() / 2; i++) {
        const float vx = poly.verts[2 * i], vy = poly.verts[2 * i + 1];
        inR = std::fmin(inR, poly.normals[2 * i] * vx + poly.normals[2 * i + 1] * vy);
        outR2 = std::fmax(outR2, vx * vx + vy * vy);
    }
    inR = std::fmax(inR, 0.0f);
    polygons.push_back(std::move(poly));
    return appendCollider(b, locX, locY, localRot, material, 2u, uint32_t(polygons.size() - 1), inR,
                          std::sqrt(outR2));
}

bool HostObjects::addCapsule(const float* d, uint32_t material, float length, float radius, uint64_t& handle,
                             std::string& err)
{
    if (!(length >= 0.0f && radius >= 0.0f)) { err = "capsule length and radius must be >= 0"; return false; }
    if (material >= materialCount()) material = 0;
    // ObjectManager::createCapsule (ObjectManager.cpp:351-388) without endpoints; calculateCapsuleInertia
    // (PhysicsGeometry.cpp:87-113) about the core's centre (centre of mass at the body origin).
    const float mass = std::fmax(0.0f, d[6]);
    const float len = std::fmax(0.0f, length), r = std::fmax(0.0f, radius);
    const float pi = float(3.14159265358979323846);
    const float rectArea = len * 2.0f * r;
    const float circleArea = pi * r * r;
    const float totalArea = rectArea + circleArea;
    const float rectMass = mass * rectArea / totalArea;
    const float capMass = mass * circleArea / totalArea;
    const float diameter = 2.0f * r;
    const float rectInertia = rectMass * (len * len + diameter * diameter) / 12.0f;
    const float dist = 4.0f * r / (3.0f * pi);
    const float capInertia = capMass * (0.5f * r * r + 0.25f * len * len + len * dist);
    const float inertia = rectInertia + capInertia + mass * 0.0f;
    const float invMass = mass == 0.0f ? 0.0f : 1.0f / mass;
    const float invInertia = inertia == 0.0f ? 0.0f : 1.0f / inertia;
    const uint32_t b = appendBody(d[0], d[1], d[3], d[4], d[2], d[5], mass, invMass, inertia, invInertia, 0.0f, 0.0f);
    const uint32_t slot = bodies[b].handleSlot;
    // createCapsuleCollider (ObjectManager.cpp:197-231): half length, radius; extents (radius, half length + radius).
    const float half = len * 0.5f;
    boxHalfW.push_back(half);
    boxHalfH.push_back(r);
    appendCollider(b, 0.0f, 0.0f, 0.0f, material, 3u, uint32_t(boxHalfW.size() - 1), r, half + r);
    handle = (uint64_t(slotGeneration[slot]) << 32) | slot;
    return true;
}

bool HostObjects::addBody(const float* d, float inertiaIn, float comX, float comY, uint64_t& handle, std::string& err)
{
    (void)err;
    const float mass = std::fmax(0.0f, d[6]);
    const float inertia = std::fmax(0.0f, inertiaIn);
    const float invMass = mass == 0.0f ? 0.0f : 1.0f / mass;
    const float invInertia = inertia == 0.0f ? 0.0f : 1.0f / inertia;
    const uint32_t b = appendBody(d[0], d[1], d[3], d[4], d[2], d[5], mass, invMass, inertia, invInertia, comX, comY);
    const uint32_t slot = bodies[b].handleSlot;
    handle = (uint64_t(slotGeneration[slot]) << 32) | slot;
    return true;
}

bool HostObjects::addCollider(uint32_t body, uint32_t type, float locX, float locY, float localRot, uint32_t material,
                              const float* p, const float* xy, uint32_t n, uint32_t& collider, std::string& err)
{
    if (body >= bodies.size()) { err = "stale body handle"; return false; }
    if (material >= materialCount()) material = 0;
    switch (type) {
    case 0: {   // createCircleCollider (:90-112)
        const float r = std::fmax(0.0f, p[0]);
        circleRadius.push_back(r);
        collider = appendCollider(body, locX, locY, localRot, material, 0u, uint32_t(circleRadius.size() - 1), r, r);
        return true;
    }
    case 1: {   // createBoxCollider (:114-139)
        const float w = std::fmax(0.0f, p[0]), h = std::fmax(0.0f, p[1]);
        const float hw = w * 0.5f, hh = h * 0.5f;
        boxHalfW.push_back(hw);
        boxHalfH.push_back(hh);
        collider = appendCollider(body, locX, locY, localRot, material, 1u, uint32_t(boxHalfW.size() - 1),
                                  std::fmin(hw, hh), std::fmax(hw, hh));
        return true;
    }
    case 3: {   // createCapsuleCollider (:197-231)
        const float len = std::fmax(0.0f, p[0]), r = std::fmax(0.0f, p[1]);
        const float half = len * 0.5f;
        boxHalfW.push_back(half);
        boxHalfH.push_back(r);
        collider = appendCollider(body, locX, locY, localRot, material, 3u, uint32_t(boxHalfW.size() - 1), r, half + r);
        return true;
    }
    case 2: {   // createPolygonCollider (:141-195): one collider per convex piece, the first returned
        if (!xy || n < 3) { err = "polygon needs at least 3 vertices"; return false; }
        std::vector<float> outline;
        if (!prepare_outline_any(xy, n, outline, err)) return false;
        std::vector<std::vector<float>> pieces = decompose_outline(outline, 16);
        if (pieces.empty()) { err = "decomposition produced no pieces"; return false; }
        collider = appendPolygonPiece(body, locX, locY, localRot, material, pieces[0]);
        for (size_t k = 1; k < pieces.size(); k++) appendPolygonPiece(body, locX, locY, localRot, material, pieces[k]);
        return true;
    }
    default: err = "unknown shape kind"; return false;
    }
}

}  // namespace ag2d

namespace ag2d {

float HostObjects::colliderArea(uint32_t c) const
{
    const HCollider& k = colliders[c];
    const float pi = float(3.14159265358979323846);
    switch (k.type) {
    case 0: { const float r = circleRadius[k.shape]; return pi * r * r; }
    case 1: return (boxHalfW[k.shape] * 2.0f) * (boxHalfH[k.shape] * 2.0f);
    case 3: {
        const float len = boxHalfW[k.shape] * 2.0f, r = boxHalfH[k.shape];
        return len * 2.0f * r + pi * r * r;
    }
    case 2: {
        const std::vector<float>& v = polygons[k.shape].verts;
        const size_t n = v.size() / 2;
        if (n < 3) return 0.0f;
        float twice = 0.0f;
        for (size_t i = 0; i < n; i++) {
            const size_t j = i + 1 == n ? 0 : i + 1;
            twice += v[2 * i] * v[2 * j + 1] - v[2 * j] * v[2 * i + 1];
        }
        return std::fmax(0.0f, twice * 0.5f);
    }
    default: return 0.0f;
    }
}

float HostObjects::colliderOwnInertia(uint32_t c, float m) const
{
    const HCollider& k = colliders[c];
    switch (k.type) {
    case 0: { const float r = circleRadius[k.shape]; return (0.5f * (r * r) + 0.0f) * m; }
    case 1: {
        const float w = boxHalfW[k.shape] * 2.0f, h = boxHalfH[k.shape] * 2.0f;
        return m * (float(1.0 / 12.0) * (w * w + h * h) + 0.0f);
    }
    case 3: {
        const float len = boxHalfW[k.shape] * 2.0f, r = boxHalfH[k.shape];
        const float pi = float(3.14159265358979323846);
        const float rectArea = len * 2.0f * r, circleArea = pi * r * r, totalArea = rectArea + circleArea;
        const float rectMass = m * rectArea / totalArea, capMass = m * circleArea / totalArea;
        const float diameter = 2.0f * r;
        const float rectInertia = rectMass * (len * len + diameter * diameter) / 12.0f;
        const float dist = 4.0f * r / (3.0f * pi);
        const float capInertia = capMass * (0.5f * r * r + 0.25f * len * len + len * dist);
        return rectInertia + capInertia + m * 0.0f;
    }
    case 2: {
        float inertia = 0.0f, cx = 0.0f, cy = 0.0f;
        polygon_inertia(m, polygons[k.shape].verts, inertia, cx, cy);
        return inertia;
    }
    default: return 0.0f;
    }
}

float HostObjects::boundRadiusOf(uint32_t b) const
{
    float radius = 0.0f;
    for (const uint32_t c : bodies[b].colliders) {
        const float x = colliders[c].comOffX, y = colliders[c].comOffY;
        radius = std::fmax(radius, std::sqrt(x * x + y * y) + colliders[c].maxExtent);
    }
    return radius;
}

}  // namespace ag2d
