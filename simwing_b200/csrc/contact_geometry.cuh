// Contact geometry on the device in FP64: closest features, the swept
// (continuous) contact query, swept AABBs and Coulomb friction, as softwing
// states them (src/softwing/contact.cpp).  Every expression keeps the
// reference's operand order, so a translation unit built without FMA
// contraction reproduces the reference's results bit for bit; the step
// kernel reuses the same functions on FP32-resident state.
#pragma once

#include "simwing_b200.h"

#include <cstdint>

namespace swb {
namespace contact {

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator-(D3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double norm2(D3 v) { return dot(v, v); }
__device__ __forceinline__ double norm(D3 v) { return sqrt(norm2(v)); }
__device__ __forceinline__ D3 unit(D3 v) {
    const double m = norm(v);
    return m > 0.0 ? v / m : D3{0.0, 0.0, 0.0};
}
__device__ __forceinline__ bool finite3(D3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }  // std::max
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }  // std::min
__device__ __forceinline__ double clamp01(double v) { return v < 0.0 ? 0.0 : (1.0 < v ? 1.0 : v); }

constexpr double kEps = 2.220446049250313e-16;  // DBL_EPSILON

// ClosestFeatureClass (contact.h:39-51)
enum : uint32_t {
    kPoint = 0, kSegmentStart, kSegmentEnd, kSegmentInterior, kTriVertex0, kTriVertex1, kTriVertex2,
    kTriEdge01, kTriEdge12, kTriEdge20, kTriFace
};

// A query result; status / features / weights as ClosestFeatureResult.
struct Closest {
    uint32_t status = SWB_GEOMETRY_UNCERTIFIABLE;
    uint32_t first_feature = kPoint, second_feature = kPoint;
    D3 first_point{0.0, 0.0, 0.0}, second_point{0.0, 0.0, 0.0};
    double fw[3] = {0.0, 0.0, 0.0}, sw[3] = {0.0, 0.0, 0.0};
    D3 normal{0.0, 0.0, 0.0};
    double distance = 0.0, gap = 0.0;
    __device__ bool certified() const { return status == SWB_GEOMETRY_CERTIFIED; }
};

__device__ __forceinline__ uint32_t segment_feature(double t) {  // contact.cpp:25-35
    const double tol = 64.0 * kEps;
    if (t <= tol) return kSegmentStart;
    if (t >= 1.0 - tol) return kSegmentEnd;
    return kSegmentInterior;
}

__device__ __forceinline__ uint32_t triangle_feature(const double w[3]) {  // contact.cpp:37-60
    const double tol = 128.0 * kEps;
    if (w[0] >= 1.0 - tol) return kTriVertex0;
    if (w[1] >= 1.0 - tol) return kTriVertex1;
    if (w[2] >= 1.0 - tol) return kTriVertex2;
    if (w[2] <= tol) return kTriEdge01;
    if (w[0] <= tol) return kTriEdge12;
    if (w[1] <= tol) return kTriEdge20;
    return kTriFace;
}

// The unit normal of the smallest-magnitude axis crossed with `d`
// (contact.cpp:62-71).
__device__ __forceinline__ D3 perpendicular(D3 d) {
    const double ax = fabs(d.x), ay = fabs(d.y), az = fabs(d.z);
    const D3 axis = (ax <= ay && ax <= az) ? D3{1.0, 0.0, 0.0}
                    : ay <= az             ? D3{0.0, 1.0, 0.0}
                                           : D3{0.0, 0.0, 1.0};
    return unit(cross(d, axis));
}

// Distance, gap, normal and certification from the two closest points
// (contact.cpp:73-93).
__device__ __forceinline__ void finish(Closest& r, D3 zero_normal, double separation) {
    const D3 diff = r.first_point - r.second_point;
    r.distance = norm(diff);
    r.gap = r.distance - separation;
    const double scale = dmax(dmax(1.0, norm(r.first_point)), norm(r.second_point));
    const double zero_tol = 64.0 * kEps * scale;
    r.normal = r.distance > zero_tol ? diff / r.distance : unit(zero_normal);
    r.status = (!finite3(r.first_point) || !finite3(r.second_point) || !finite3(r.normal) ||
                !isfinite(r.distance) || !isfinite(r.gap) || norm2(r.normal) == 0.0)
                   ? SWB_GEOMETRY_UNCERTIFIABLE
                   : SWB_GEOMETRY_CERTIFIED;
}

__device__ __forceinline__ bool valid_separation(double s) { return isfinite(s) && s >= 0.0; }

// Closest point of triangle (a, b, c) to `p` by Voronoi regions
// (closestVertexTriangle, contact.cpp:141-245).
static __device__ __noinline__ Closest closest_vertex_triangle(D3 p, D3 a, D3 b, D3 c, double separation) {
    Closest r;
    r.first_feature = kPoint;
    r.first_point = p;
    r.fw[0] = 1.0;
    if (!finite3(p) || !finite3(a) || !finite3(b) || !finite3(c) || !isfinite(separation)) {
        r.status = SWB_GEOMETRY_NON_FINITE;
        return r;
    }
    if (!valid_separation(separation)) return r;
    const D3 ab = b - a, ac = c - a, bc = c - b;
    const double scale2 = dmax(dmax(norm2(ab), norm2(ac)), norm2(bc));
    const D3 area_normal = cross(ab, ac);
    const double area2 = norm2(area_normal);
    const double rel = 64.0 * kEps;
    if (!(scale2 > 0.0) || !(area2 > rel * rel * scale2 * scale2)) {
        r.status = SWB_GEOMETRY_DEGENERATE;
        return r;
    }
    const D3 ap = p - a;
    const double d1 = dot(ab, ap), d2 = dot(ac, ap);
    double* w = r.sw;
    if (d1 <= 0.0 && d2 <= 0.0) {
        r.second_point = a;
        w[0] = 1.0; w[1] = 0.0; w[2] = 0.0;
    } else {
        const D3 bp = p - b;
        const double d3 = dot(ab, bp), d4 = dot(ac, bp);
        if (d3 >= 0.0 && d4 <= d3) {
            r.second_point = b;
            w[0] = 0.0; w[1] = 1.0; w[2] = 0.0;
        } else {
            const double vc = d1 * d4 - d3 * d2;
            if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) {
                const double t = d1 / (d1 - d3);
                r.second_point = a + t * ab;
                w[0] = 1.0 - t; w[1] = t; w[2] = 0.0;
            } else {
                const D3 cp = p - c;
                const double d5 = dot(ab, cp), d6 = dot(ac, cp);
                if (d6 >= 0.0 && d5 <= d6) {
                    r.second_point = c;
                    w[0] = 0.0; w[1] = 0.0; w[2] = 1.0;
                } else {
                    const double vb = d5 * d2 - d1 * d6;
                    if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) {
                        const double t = d2 / (d2 - d6);
                        r.second_point = a + t * ac;
                        w[0] = 1.0 - t; w[1] = 0.0; w[2] = t;
                    } else {
                        const double va = d3 * d6 - d5 * d4;
                        if (va <= 0.0 && d4 - d3 >= 0.0 && d5 - d6 >= 0.0) {
                            const double t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
                            r.second_point = b + t * (c - b);
                            w[0] = 0.0; w[1] = 1.0 - t; w[2] = t;
                        } else {
                            const double inv = 1.0 / (va + vb + vc);
                            const double v = vb * inv, u = vc * inv;
                            w[0] = 1.0 - v - u; w[1] = v; w[2] = u;
                            r.second_point = w[0] * a + w[1] * b + w[2] * c;
                        }
                    }
                }
            }
        }
    }
    r.second_feature = triangle_feature(r.sw);
    finish(r, area_normal, separation);
    return r;
}

// Closest points of two segments (closestEdgeEdge, contact.cpp:247-304).
static __device__ __noinline__ Closest closest_edge_edge(D3 p0, D3 p1, D3 q0, D3 q1, double separation) {
    Closest r;
    if (!finite3(p0) || !finite3(p1) || !finite3(q0) || !finite3(q1) || !isfinite(separation)) {
        r.status = SWB_GEOMETRY_NON_FINITE;
        return r;
    }
    if (!valid_separation(separation)) return r;
    const D3 u = p1 - p0, v = q1 - q0, w0 = p0 - q0;
    const double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w0), e = dot(v, w0);
    if (!(a > 0.0) || !(c > 0.0)) {
        r.status = SWB_GEOMETRY_DEGENERATE;
        return r;
    }
    const double den = a * c - b * b;
    const double parallel_tol = 64.0 * kEps * a * c;
    double s = 0.0;
    if (den > parallel_tol) s = clamp01((b * e - c * d) / den);
    double t = (b * s + e) / c;
    if (t < 0.0) {
        t = 0.0;
        s = clamp01(-d / a);
    } else if (t > 1.0) {
        t = 1.0;
        s = clamp01((b - d) / a);
    }
    r.first_point = p0 + s * u;
    r.second_point = q0 + t * v;
    r.fw[0] = 1.0 - s; r.fw[1] = s; r.fw[2] = 0.0;
    r.sw[0] = 1.0 - t; r.sw[1] = t; r.sw[2] = 0.0;
    r.first_feature = segment_feature(s);
    r.second_feature = segment_feature(t);
    D3 zero_normal = cross(u, v);
    if (norm2(zero_normal) <= parallel_tol) zero_normal = perpendicular(u);
    finish(r, zero_normal, separation);
    return r;
}

// A primitive moving linearly over the substep: up to three points.
struct Linear {
    D3 prev[3];
    D3 cur[3];
    int count;
};

__device__ __forceinline__ Closest evaluate_at(uint32_t kind, const Linear& f, const Linear& s, double time,
                                               double separation) {
    D3 a[3], b[3];
    for (int i = 0; i < f.count; ++i) a[i] = f.prev[i] + time * (f.cur[i] - f.prev[i]);
    for (int i = 0; i < s.count; ++i) b[i] = s.prev[i] + time * (s.cur[i] - s.prev[i]);
    if (kind == SWB_FEATURE_VERTEX_TRIANGLE) return closest_vertex_triangle(a[0], b[0], b[1], b[2], separation);
    return closest_edge_edge(a[0], a[1], b[0], b[1], separation);
}

__device__ __forceinline__ Closest evaluate_current(uint32_t kind, const Linear& f, const Linear& s,
                                                    double separation) {
    if (kind == SWB_FEATURE_VERTEX_TRIANGLE) return closest_vertex_triangle(f.cur[0], s.cur[0], s.cur[1], s.cur[2], separation);
    return closest_edge_edge(f.cur[0], f.cur[1], s.cur[0], s.cur[1], separation);
}

struct Ccd {
    uint32_t state = SWB_CCD_INDETERMINATE;
    double toi = 0.0, lower = 0.0, upper = 1.0;
    Closest geometry;
    int iterations = 0, subdivisions = 0;
    bool fallback = false;
};

// One pending interval of the fallback search: its ends and the distances
// there (the geometry at `lower` is re-evaluated when needed; the query is a
// pure function of time, so it is the same value the search saw).
struct Interval {
    double lower, upper, lower_distance, upper_distance;
};

// Bisection of [safe, impact] to the time tolerance (sweptContact's
// refineImpact, contact.cpp:778-804).  Returns false on an uncertifiable
// midpoint (state Indeterminate).
//
// A tolerance below the spacing of doubles near the impact time lets the
// midpoint round onto an end of the interval.  When the update then leaves
// the interval as it was, every later pass would evaluate the same midpoint
// and change nothing again (the reference's loop spins there for good), so
// the search stops with the interval it has.  Wherever the reference's loop
// ends, every pass changes the interval and the result is the same.  A pass
// that changes the interval roughly halves it, so the search takes at most
// about 1,100 passes; kMaxRefinePasses bounds it regardless.
constexpr int kMaxRefinePasses = 4096;

__device__ __forceinline__ bool refine_impact(uint32_t kind, const Linear& f, const Linear& s, double separation,
                                              const swb_ccd_settings& cs, double safe, double impact,
                                              Closest impact_geometry, Ccd& out) {
    double lower = safe, upper = impact;
    for (int pass = 0; upper - lower > cs.time_tolerance && pass < kMaxRefinePasses; ++pass) {
        const double middle = 0.5 * (lower + upper);
        const Closest g = evaluate_at(kind, f, s, middle, separation);
        if (!g.certified()) {
            out.state = SWB_CCD_INDETERMINATE;
            out.geometry = g;
            return false;
        }
        const double was_lower = lower, was_upper = upper;
        if (g.gap <= cs.distance_tolerance) {
            upper = middle;
            impact_geometry = g;
        } else {
            lower = middle;
        }
        if (lower == was_lower && upper == was_upper) break;
    }
    out.state = SWB_CCD_IMPACT;
    out.toi = upper;
    out.lower = lower;
    out.upper = upper;
    out.geometry = impact_geometry;
    return true;
}

// Continuous contact over the substep: conservative advancement, then an
// interval subdivision fallback (sweptContact, contact.cpp:669-945).
// `queue` holds interval_subdivisions + 1 entries of scratch.
static __device__ __noinline__ Ccd swept_contact(uint32_t kind, const Linear& f, const Linear& s, double separation,
                                          const swb_ccd_settings& cs, Interval* queue) {
    Ccd r;
    const bool counts = (kind == SWB_FEATURE_VERTEX_TRIANGLE && f.count == 1 && s.count == 3) ||
                        (kind == SWB_FEATURE_EDGE_EDGE && f.count == 2 && s.count == 2);
    if (!counts || !valid_separation(separation) || cs.conservative_iterations < 0 ||
        cs.interval_subdivisions < 0 || !isfinite(cs.time_tolerance) || !(cs.time_tolerance > 0.0) ||
        !isfinite(cs.distance_tolerance) || !(cs.distance_tolerance > 0.0))
        return r;
    for (int i = 0; i < f.count; ++i)
        if (!finite3(f.prev[i]) || !finite3(f.cur[i])) return r;
    for (int i = 0; i < s.count; ++i)
        if (!finite3(s.prev[i]) || !finite3(s.cur[i])) return r;
    double first_speed = 0.0, second_speed = 0.0;
    for (int i = 0; i < f.count; ++i) first_speed = dmax(first_speed, norm(f.cur[i] - f.prev[i]));
    for (int i = 0; i < s.count; ++i) second_speed = dmax(second_speed, norm(s.cur[i] - s.prev[i]));
    const double speed = first_speed + second_speed;
    const double tol = cs.distance_tolerance;

    const Closest initial = evaluate_at(kind, f, s, 0.0, separation);
    if (!initial.certified()) {
        r.geometry = initial;
        return r;
    }
    if (initial.gap <= tol) {
        r.state = SWB_CCD_INITIALLY_PROXIMATE;
        r.toi = 0.0; r.lower = 0.0; r.upper = 0.0;
        r.geometry = initial;
        return r;
    }
    if (!(speed > 0.0)) {
        r.state = SWB_CCD_NO_IMPACT;
        r.toi = 1.0; r.lower = 1.0; r.upper = 1.0;
        r.geometry = initial;
        return r;
    }
    if (cs.conservative_iterations == 0 && cs.interval_subdivisions == 0) {
        r.geometry = initial;
        return r;
    }

    double time = 0.0;
    Closest current = initial;
    bool fallback = false;
    for (int it = 0; it < cs.conservative_iterations; ++it) {
        ++r.iterations;
        const double safe_gap = current.gap - tol;
        const double advance = 0.9 * safe_gap / speed;
        if (!(advance > 0.0) || !isfinite(advance)) {
            fallback = true;
            break;
        }
        const double next = time + advance;
        if (next >= 1.0) {
            const double lower_bound = current.distance - speed * (1.0 - time);
            if (lower_bound > separation + tol) {
                r.state = SWB_CCD_NO_IMPACT;
                r.toi = 1.0; r.lower = time; r.upper = 1.0;
                r.geometry = evaluate_at(kind, f, s, 1.0, separation);
                if (!r.geometry.certified()) r.state = SWB_CCD_INDETERMINATE;
                return r;
            }
            const Closest end = evaluate_at(kind, f, s, 1.0, separation);
            if (!end.certified()) {
                r.geometry = end;
                return r;
            }
            if (end.gap <= tol) {
                refine_impact(kind, f, s, separation, cs, time, 1.0, end, r);
                return r;
            }
            fallback = true;
            break;
        }
        const Closest g = evaluate_at(kind, f, s, next, separation);
        if (!g.certified()) {
            r.geometry = g;
            return r;
        }
        if (g.gap <= tol) {
            refine_impact(kind, f, s, separation, cs, time, next, g, r);
            return r;
        }
        time = next;
        current = g;
    }
    if (r.iterations >= cs.conservative_iterations) fallback = true;
    if (!fallback || cs.interval_subdivisions == 0) {
        r.geometry = current;
        return r;
    }

    r.fallback = true;
    const Closest end = evaluate_at(kind, f, s, 1.0, separation);
    if (!end.certified()) {
        r.geometry = end;
        return r;
    }
    if (end.gap <= tol) {
        refine_impact(kind, f, s, separation, cs, 0.0, 1.0, end, r);
        r.fallback = true;
        return r;
    }
    // First-in first-out ring of pending intervals; at most
    // interval_subdivisions + 1 are pending at once.
    const int capacity = cs.interval_subdivisions + 1;
    int head = 0, size = 0;
    queue[0] = {0.0, 1.0, initial.distance, end.distance};
    size = 1;
    while (size > 0) {
        const Interval iv = queue[head];
        head = head + 1 == capacity ? 0 : head + 1;
        --size;
        const double width = iv.upper - iv.lower;
        const double certified_lower = 0.5 * (iv.lower_distance + iv.upper_distance - speed * width);
        if (certified_lower > separation + tol) continue;
        if (r.subdivisions >= cs.interval_subdivisions) {
            r.geometry = evaluate_at(kind, f, s, iv.lower, separation);
            return r;
        }
        const double middle = 0.5 * (iv.lower + iv.upper);
        const Closest m = evaluate_at(kind, f, s, middle, separation);
        ++r.subdivisions;
        if (!m.certified()) {
            r.geometry = m;
            return r;
        }
        if (m.gap <= tol) {
            refine_impact(kind, f, s, separation, cs, iv.lower, middle, m, r);
            r.fallback = true;
            return r;
        }
        int tail = head + size;
        if (tail >= capacity) tail -= capacity;
        queue[tail] = {iv.lower, middle, iv.lower_distance, m.distance};
        tail = tail + 1 == capacity ? 0 : tail + 1;
        queue[tail] = {middle, iv.upper, m.distance, iv.upper_distance};
        size += 2;
    }
    r.state = SWB_CCD_NO_IMPACT;
    r.toi = 1.0; r.lower = 1.0; r.upper = 1.0;
    r.geometry = end;
    return r;
}

// Swept AABB of a primitive's points, expanded by `expansion` plus a
// coordinate-relative margin (sweptExpandedAabb, contact.cpp:488-526).
struct Box {
    double lo[3], hi[3];
};
__device__ __forceinline__ Box swept_box(const D3* prev, const D3* cur, int count, double expansion) {
    Box b{{prev[0].x, prev[0].y, prev[0].z}, {prev[0].x, prev[0].y, prev[0].z}};
    double scale = 1.0;
    auto include = [&](D3 p) {
        b.lo[0] = dmin(b.lo[0], p.x); b.lo[1] = dmin(b.lo[1], p.y); b.lo[2] = dmin(b.lo[2], p.z);
        b.hi[0] = dmax(b.hi[0], p.x); b.hi[1] = dmax(b.hi[1], p.y); b.hi[2] = dmax(b.hi[2], p.z);
        scale = dmax(dmax(dmax(scale, fabs(p.x)), fabs(p.y)), fabs(p.z));
    };
    for (int i = 0; i < count; ++i) {
        include(prev[i]);
        include(cur[i]);
    }
    const double margin = 64.0 * kEps * dmax(scale, expansion);
    const double total = expansion + margin;
    for (int k = 0; k < 3; ++k) {
        b.lo[k] -= total;
        b.hi[k] += total;
    }
    return b;
}

__device__ __forceinline__ bool boxes_overlap(const Box& a, const Box& b) {
    return a.lo[0] <= b.hi[0] && b.lo[0] <= a.hi[0] && a.lo[1] <= b.hi[1] && b.lo[1] <= a.hi[1] &&
           a.lo[2] <= b.hi[2] && b.lo[2] <= a.hi[2];
}

// One candidate row scanned by a warp (all 32 lanes call it).  Row r < nv:
// the vertex-triangle features of surface vertex r against every triangle
// not holding it, in triangle order; row nv + i: the edge-edge features of
// edge i with every later edge sharing no node, in edge order.  Node
// identities are whatever the id arrays hold (node indices or slots).
// emit(col, k) is called by the hitting lane for its k-th hit of the row, in
// column order; returns the row's hit count.
template <class Emit>
__device__ __forceinline__ uint32_t scan_candidate_row(uint32_t row, uint32_t nv, uint32_t ne, uint32_t nt,
                                                       const uint32_t* __restrict__ vid,
                                                       const uint2* __restrict__ eid,
                                                       const uint3* __restrict__ tid3, const Box* __restrict__ vbox,
                                                       const Box* __restrict__ ebox, const Box* __restrict__ tbox,
                                                       Emit emit) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t hits = 0;
    if (row < nv) {
        const uint32_t v = vid[row];
        const Box b = vbox[row];
        for (uint32_t c0 = 0; c0 < nt; c0 += 32) {
            const uint32_t t = c0 + lane;
            bool hit = false;
            if (t < nt) {
                const uint3 tri = tid3[t];
                hit = tri.x != v && tri.y != v && tri.z != v && boxes_overlap(b, tbox[t]);
            }
            const unsigned mask = __ballot_sync(0xffffffffu, hit);
            if (hit) emit(t, hits + __popc(mask & ((1u << lane) - 1u)));
            hits += __popc(mask);
        }
    } else {
        const uint32_t i = row - nv;
        const uint2 e = eid[i];
        const Box b = ebox[i];
        for (uint32_t c0 = i + 1; c0 < ne; c0 += 32) {
            const uint32_t j = c0 + lane;
            bool hit = false;
            if (j < ne) {
                const uint2 f = eid[j];
                hit = e.x != f.x && e.x != f.y && e.y != f.x && e.y != f.y && boxes_overlap(b, ebox[j]);
            }
            const unsigned mask = __ballot_sync(0xffffffffu, hit);
            if (hit) emit(j, hits + __popc(mask & ((1u << lane) - 1u)));
            hits += __popc(mask);
        }
    }
    return hits;
}

// ContactFrictionState (contact.h:178-182)
enum : uint32_t { kFrictionInactive = 0, kFrictionSticking = 1, kFrictionSliding = 2 };

struct Friction {
    uint32_t state = kFrictionInactive;
    D3 initial_tangent{0.0, 0.0, 0.0}, final_tangent{0.0, 0.0, 0.0}, impulse{0.0, 0.0, 0.0};
    double cone_ratio = 0.0, work = 0.0;
};

// Velocity-level Coulomb friction of one contact (solveCoulombFriction,
// contact.cpp:434-486).
__device__ __forceinline__ Friction coulomb_friction(D3 relative_velocity, D3 normal, double inv_mass,
                                                     double normal_impulse, double static_mu,
                                                     double dynamic_mu, bool active) {
    Friction r;
    if (!finite3(relative_velocity) || !finite3(normal) || !isfinite(inv_mass) || !isfinite(normal_impulse) ||
        !isfinite(static_mu) || !isfinite(dynamic_mu) || !(inv_mass > 0.0) || normal_impulse < 0.0 ||
        dynamic_mu < 0.0 || static_mu < dynamic_mu || fabs(norm2(normal) - 1.0) > 1.0e-8)
        return r;
    r.initial_tangent = relative_velocity - dot(relative_velocity, normal) * normal;
    r.final_tangent = r.initial_tangent;
    const double speed = norm(r.initial_tangent);
    if (!active || !(normal_impulse > 0.0) || !(speed > 0.0)) return r;
    const D3 stop = -r.initial_tangent / inv_mass;
    const double stop_magnitude = norm(stop);
    const double static_limit = static_mu * normal_impulse;
    if (stop_magnitude <= static_limit) {
        r.state = kFrictionSticking;
        r.impulse = stop;
    } else {
        r.state = kFrictionSliding;
        const double applied = dmin(dynamic_mu * normal_impulse, stop_magnitude);
        r.impulse = -applied * (r.initial_tangent / speed);
    }
    r.final_tangent = r.initial_tangent + inv_mass * r.impulse;
    const double magnitude = norm(r.impulse);
    r.cone_ratio = static_limit > 0.0 ? magnitude / static_limit : 0.0;
    r.work = dot(r.impulse, r.initial_tangent) + 0.5 * inv_mass * norm2(r.impulse);
    return r;
}

}  // namespace contact
}  // namespace swb
