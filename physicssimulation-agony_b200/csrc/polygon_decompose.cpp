// Concave polygon outlines split into convex pieces, as the reference engine does at polygon creation
// (PhysicsGeometry::decomposeConcave and limitConvexPieceVertexCount, SimulationImpl/PolygonDecomposition.cpp:
// 704-736, 758-831) with its default methods: Bayazit's diagonal splitting with merging of the pieces, ear clipping
// when no valid diagonal exists, and the fan split of pieces above the vertex limit. The arithmetic follows the
// reference's expression order in single precision so the pieces are the reference's bit for bit; the product calls
// this on the host, once per created polygon.
#include "host_objects.hpp"

#include <algorithm>
#include <cmath>
#include <limits>
#include <optional>

namespace ag2d {
namespace {

struct V2 {
    float x, y;
};
using Poly = std::vector<V2>;

constexpr float kEps = 1e-9f;          // kConvexEpsilon (:12)
constexpr float kTouchSq = 1e-12f;     // kTouchEpsSq (:78)

inline float cross(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }
inline float turn(V2 a, V2 b, V2 c) { return (b.x - a.x) * (c.y - a.y) - (b.y - a.y) * (c.x - a.x); }
inline V2 sub(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
inline float dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline float length(V2 a) { return std::sqrt(dot(a, a)); }

float signed_area(const Poly& p)   // polygonArea (:24-36)
{
    const size_t n = p.size();
    if (n < 3) return 0.0f;
    float s = 0.0f;
    for (size_t i = 0; i < n; i++) {
        const V2 a = p[i], b = p[(i + 1) % n];
        s += a.x * b.y - b.x * a.y;
    }
    return s * 0.5f;
}

bool reflex(V2 prev, V2 cur, V2 next) { return turn(prev, cur, next) < -kEps; }

bool convex(const Poly& p)   // isConvexPolygon (:618-634)
{
    const size_t n = p.size();
    if (n < 4) return true;
    for (size_t i = 0; i < n; i++)
        if (turn(p[(i + n - 1) % n], p[i], p[(i + 1) % n]) < -kEps) return false;
    return true;
}

bool inside(V2 q, const Poly& p)   // even-odd crossing test (pointInPolygon, :43-61)
{
    bool in = false;
    const size_t n = p.size();
    for (size_t i = 0; i < n; i++) {
        const V2 a = p[i], b = p[(i + 1) % n];
        if ((a.y > q.y) != (b.y > q.y)) {
            const float xCross = (b.x - a.x) * (q.y - a.y) / (b.y - a.y + 1e-12f) + a.x;
            if (q.x < xCross) in = !in;
        }
    }
    return in;
}

bool proper_cross(V2 a, V2 b, V2 c, V2 d)   // segmentsIntersect (:63-76): strict crossings only
{
    const float s1 = turn(a, b, c), s2 = turn(a, b, d), s3 = turn(c, d, a), s4 = turn(c, d, b);
    return ((s1 > kEps && s2 < -kEps) || (s1 < -kEps && s2 > kEps)) &&
           ((s3 > kEps && s4 < -kEps) || (s3 < -kEps && s4 > kEps));
}

float seg_dist_sq(V2 p, V2 a, V2 b)   // pointSegDistSq (:80-88)
{
    const V2 ab = sub(b, a);
    const float len2 = dot(ab, ab);
    float t = len2 > 0.0f ? dot(sub(p, a), ab) / len2 : 0.0f;
    t = std::clamp(t, 0.0f, 1.0f);
    const V2 foot = {a.x + ab.x * t, a.y + ab.y * t};
    const V2 d = sub(p, foot);
    return dot(d, d);
}

// The diagonal's direction lies strictly inside the corner at vertex k (both sides for a convex corner, either
// side for a reflex one): the cone tests of isValidDiagonal (:108-142).
bool in_cone(const Poly& p, size_t k, V2 toward)
{
    const size_t n = p.size();
    const V2 prev = p[(k + n - 1) % n], cur = p[k], next = p[(k + 1) % n];
    const V2 dir = sub(toward, cur), vin = sub(next, cur), vout = sub(prev, cur);
    const bool a = cross(vin, dir) <= kEps, b = cross(dir, vout) <= kEps;
    return reflex(prev, cur, next) ? !(a && b) : !(a || b);
}

bool valid_diagonal(const Poly& p, size_t i, size_t j)   // isValidDiagonal (:90-144)
{
    const size_t n = p.size();
    if (i == j || (i + 1) % n == j || (j + 1) % n == i) return false;
    const V2 pi = p[i], pj = p[j];
    for (size_t k = 0; k < n; k++) {
        const size_t k1 = (k + 1) % n;
        if (k != i && k != j && seg_dist_sq(p[k], pi, pj) <= kTouchSq) return false;
        if (k == i || k == j || k1 == i || k1 == j) continue;
        if (proper_cross(pi, pj, p[k], p[k1])) return false;
    }
    const V2 mid = {(pi.x + pj.x) * 0.5f, (pi.y + pj.y) * 0.5f};
    if (!inside(mid, p)) return false;
    return in_cone(p, i, pj) && in_cone(p, j, pi);
}

Poly hull(const Poly& pts)   // convexHull2D (:146-197): Andrew's monotone chain after a 1e-7 dedupe
{
    Poly pt;
    for (const V2& q : pts) {
        bool seen = false;
        for (const V2& c : pt)
            if (length(sub(q, c)) < 1e-7f) { seen = true; break; }
        if (!seen) pt.push_back(q);
    }
    if (pt.size() < 3) return pt;
    std::sort(pt.begin(), pt.end(), [](const V2& a, const V2& b) { return a.x != b.x ? a.x < b.x : a.y < b.y; });
    auto chain = [](auto first, auto last) {
        Poly c;
        for (auto it = first; it != last; ++it) {
            while (c.size() >= 2 && cross(sub(c.back(), c[c.size() - 2]), sub(*it, c.back())) <= 1e-9f) c.pop_back();
            c.push_back(*it);
        }
        c.pop_back();
        return c;
    };
    Poly lower = chain(pt.begin(), pt.end());
    const Poly upper = chain(pt.rbegin(), pt.rend());
    lower.insert(lower.end(), upper.begin(), upper.end());
    return lower;
}

// Two convex pieces merge when the hull of their vertices has their summed area (tryMergeConvex, :199-218);
// repeated over all pairs, first pair first, until none merges (mergeConvexPolygons, :220-253).
std::vector<Poly> merge_pieces(std::vector<Poly> in)
{
    if (in.size() <= 1) return in;
    std::vector<Poly> ps;
    for (Poly& p : in)
        if (std::abs(signed_area(p)) > 1e-8f) ps.push_back(std::move(p));
    for (bool merged = true; merged;) {
        merged = false;
        for (size_t i = 0; i < ps.size() && !merged; i++)
            for (size_t j = i + 1; j < ps.size() && !merged; j++) {
                const float a = std::abs(signed_area(ps[i])), b = std::abs(signed_area(ps[j]));
                if (a < 1e-8f || b < 1e-8f) continue;
                Poly both = ps[i];
                both.insert(both.end(), ps[j].begin(), ps[j].end());
                Poly h = hull(both);
                if (std::abs(std::abs(signed_area(h)) - (a + b)) < 1e-6f) {
                    ps[i] = std::move(h);
                    ps.erase(ps.begin() + j);
                    merged = true;
                }
            }
    }
    return ps;
}

// Bayazit (tryBayazitRec, :259-322): at the first reflex vertex, split along the shortest valid diagonal and
// recurse into both halves; nullopt when some reflex vertex has no valid diagonal.
std::optional<std::vector<Poly>> bayazit(const Poly& p)
{
    const size_t n = p.size();
    if (n <= 3 || convex(p)) return std::vector<Poly>{p};
    int r = -1;
    for (size_t i = 0; i < n && r < 0; i++)
        if (reflex(p[(i + n - 1) % n], p[i], p[(i + 1) % n])) r = int(i);
    if (r < 0) return std::vector<Poly>{p};
    const int nn = int(n);
    int best = -1;
    float bestDist = std::numeric_limits<float>::max();
    for (int j = 0; j < nn; j++) {
        if (j == r || j == (r - 1 + nn) % nn || j == (r + 1) % nn) continue;
        if (!valid_diagonal(p, size_t(r), size_t(j))) continue;
        const float d = length(sub(p[j], p[r]));
        if (d < bestDist) { bestDist = d; best = j; }
    }
    if (best < 0) return std::nullopt;
    const int lo = std::min(r, best), hi = std::max(r, best);
    const Poly first(p.begin() + lo, p.begin() + hi + 1);
    Poly second(p.begin() + hi, p.end());
    second.insert(second.end(), p.begin(), p.begin() + lo + 1);
    auto a = bayazit(first);
    if (!a) return std::nullopt;
    auto b = bayazit(second);
    if (!b) return std::nullopt;
    a->insert(a->end(), b->begin(), b->end());
    return a;
}

// Ear clipping over vertex indices (triangulateEarClip, :502-555): the first convex corner whose triangle holds
// no other vertex is cut off; with no ear left the rest is fanned from its first vertex.
bool in_triangle(V2 q, V2 a, V2 b, V2 c)   // pointInTriangle (:474-482), boundary included
{
    const float d1 = turn(a, b, q), d2 = turn(b, c, q), d3 = turn(c, a, q);
    const bool neg = d1 < 0.0f || d2 < 0.0f || d3 < 0.0f, pos = d1 > 0.0f || d2 > 0.0f || d3 > 0.0f;
    return !(neg && pos);
}

std::vector<std::vector<int>> ear_clip(std::vector<int> ring, const Poly& v)
{
    std::vector<std::vector<int>> tris;
    while (ring.size() > 3) {
        const size_t n = ring.size();
        bool cut = false;
        for (size_t i = 0; i < n && !cut; i++) {
            const size_t ip = (i + n - 1) % n, in = (i + 1) % n;
            const V2 a = v[ring[ip]], b = v[ring[i]], c = v[ring[in]];
            if (turn(a, b, c) <= kEps) continue;
            bool blocked = false;
            for (size_t k = 0; k < n && !blocked; k++)
                if (k != ip && k != i && k != in && in_triangle(v[ring[k]], a, b, c)) blocked = true;
            if (blocked) continue;
            tris.push_back({ring[ip], ring[i], ring[in]});
            ring.erase(ring.begin() + long(i));
            cut = true;
        }
        if (!cut) {
            for (size_t i = 1; i + 1 < ring.size(); i++) tris.push_back({ring[0], ring[i], ring[i + 1]});
            ring.clear();
        }
    }
    if (ring.size() == 3) tris.push_back(ring);
    return tris;
}

bool convex_indexed(const std::vector<int>& ring, const Poly& v)   // isConvexIndexed (:484-500)
{
    const size_t n = ring.size();
    if (n < 4) return true;
    for (size_t i = 0; i < n; i++)
        if (turn(v[ring[(i + n - 1) % n]], v[ring[i]], v[ring[(i + 1) % n]]) < -kEps) return false;
    return true;
}

// Pieces sharing an edge (a's edge i..i+1 is b's j+1..j) merge while the union stays convex, first pair first
// (findSharedEdge, mergeAcrossEdge, mergeConvexPieces: :557-616).
void merge_across_edges(std::vector<std::vector<int>>& ps, const Poly& v)
{
    for (bool changed = true; changed;) {
        changed = false;
        for (size_t a = 0; a < ps.size() && !changed; a++)
            for (size_t b = a + 1; b < ps.size() && !changed; b++) {
                const std::vector<int>& A = ps[a];
                const std::vector<int>& B = ps[b];
                const size_t na = A.size(), nb = B.size();
                size_t ea = 0, eb = 0;
                bool shared = false;
                for (size_t i = 0; i < na && !shared; i++)
                    for (size_t j = 0; j < nb && !shared; j++)
                        if (B[j] == A[(i + 1) % na] && B[(j + 1) % nb] == A[i]) { ea = i; eb = j; shared = true; }
                if (!shared) continue;
                std::vector<int> m(A.begin(), A.begin() + long(ea) + 1);
                for (size_t c = 0; c + 2 < nb; c++) m.push_back(B[(eb + 2 + c) % nb]);
                m.insert(m.end(), A.begin() + long(ea) + 1, A.end());
                if (!convex_indexed(m, v)) continue;
                ps[a] = std::move(m);
                ps.erase(ps.begin() + long(b));
                changed = true;
            }
    }
}

std::vector<Poly> ear_clip_pieces(const Poly& v)   // decomposeConcaveEarClipping (:673-691)
{
    std::vector<int> ring(v.size());
    for (size_t i = 0; i < ring.size(); i++) ring[i] = int(i);
    std::vector<std::vector<int>> ps = ear_clip(std::move(ring), v);
    merge_across_edges(ps, v);
    std::vector<Poly> out;
    for (const std::vector<int>& p : ps) {
        Poly q;
        for (const int k : p) q.push_back(v[k]);
        out.push_back(std::move(q));
    }
    return out;
}

Poly to_poly(const std::vector<float>& xy)
{
    Poly p(xy.size() / 2);
    for (size_t i = 0; i < p.size(); i++) p[i] = {xy[2 * i], xy[2 * i + 1]};
    return p;
}

std::vector<float> to_xy(const Poly& p)
{
    std::vector<float> xy(p.size() * 2);
    for (size_t i = 0; i < p.size(); i++) { xy[2 * i] = p[i].x; xy[2 * i + 1] = p[i].y; }
    return xy;
}

}  // namespace

bool outline_is_convex(const std::vector<float>& xy) { return convex(to_poly(xy)); }

bool outline_is_simple(const std::vector<float>& xy)   // isSimplePolygon (PolygonDecomposition.cpp:636-671)
{
    const Poly v = to_poly(xy);
    const size_t n = v.size();
    if (n < 3) return false;
    for (size_t i = 0; i < n; i++) {   // spikes: a reversal along the vertex's own edge
        const V2 e1 = sub(v[i], v[(i + n - 1) % n]), e2 = sub(v[(i + 1) % n], v[i]);
        if (dot(e1, e2) < 0.0f && std::abs(cross(e1, e2)) <= 1e-6f * length(e1) * length(e2)) return false;
    }
    for (size_t i = 0; i < n; i++) {
        const V2 a = v[i], b = v[(i + 1) % n];
        for (size_t j = i + 1; j < n; j++) {
            if (j == i + 1 || (i == 0 && j == n - 1)) continue;
            const V2 c = v[j], d = v[(j + 1) % n];
            if (proper_cross(a, b, c, d)) return false;
            if (seg_dist_sq(a, c, d) <= kTouchSq || seg_dist_sq(b, c, d) <= kTouchSq ||
                seg_dist_sq(c, a, b) <= kTouchSq || seg_dist_sq(d, a, b) <= kTouchSq)
                return false;
        }
    }
    return true;
}

std::vector<std::vector<float>> decompose_outline(const std::vector<float>& xy, size_t maxVertices)
{
    const Poly v = to_poly(xy);
    std::vector<Poly> pieces;
    if (v.size() < 3) return {};
    if (convex(v)) {
        pieces.push_back(v);
    } else if (auto b = bayazit(v)) {   // decomposeConcave, Bayazit first (:704-736)
        pieces = merge_pieces(std::move(*b));
    } else {
        pieces = ear_clip_pieces(v);
    }
    // limitConvexPieceVertexCount with the fan split (:758-783, 811-831): a piece above the limit becomes fans
    // from its first vertex, consecutive fans sharing an edge.
    maxVertices = std::max<size_t>(maxVertices, 3);
    std::vector<std::vector<float>> out;
    for (const Poly& p : pieces) {
        const size_t n = p.size();
        if (n <= maxVertices) { out.push_back(to_xy(p)); continue; }
        for (size_t start = 1;;) {
            const size_t end = std::min(start + maxVertices - 2, n - 1);
            Poly f{p[0]};
            f.insert(f.end(), p.begin() + long(start), p.begin() + long(end) + 1);
            out.push_back(to_xy(f));
            if (end == n - 1) break;
            start = end;
        }
    }
    return out;
}

}  // namespace ag2d
