/*
 * ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product.
 *
 * Plain-C, FP64 restatement of the reference XPBD structure step on the
 * path the device solver covers.  Each function follows the reference
 * arithmetic operation for operation (same expression trees, FP contraction
 * off) so that on the same inputs it reproduces the reference's own serial
 * solver bit for bit; tests pin it against the reference compiled from
 * source (oracle/_ref) and against the reference's known-answer tests.
 *
 *   swo_step           SoftBody::step / stepCoupled      soft_body.cpp:981-1070
 *   substep            integrateSubstep(+Trial)          soft_body.cpp:1072-1460
 *   pressure_scatter   accumulatePressureForces (serial) soft_body.cpp:1492-1509
 *   predict            predictPositions                  soft_body.cpp:1536-1566
 *   finalize           finalizeVelocities                soft_body.cpp:1568-1585
 *   project_distance   projectDistanceConstraint         soft_body.cpp:1598-1640
 *   evaluate_dihedral  evaluateDihedral                  soft_body.cpp:1648-1711
 *   solve_dihedral     solveDihedralConstraint           soft_body.cpp:1754-1792
 *   measure/restore_momentum                             soft_body.cpp:119-190
 *   load_path_order    loadPathConstraintOrder           soft_body.cpp:528-629
 *   cable_pair         solveCablePair (+ distribution)   soft_body.cpp:1265-1317, 1380-1388
 *   membrane_setup     addMembraneElements               soft_body.cpp:664-690
 *   membrane_strain    evaluateMembraneElement (strain)  soft_body.cpp:204-270
 *   solve_membrane     membraneElementCorrections +
 *                      solveMembraneElement              soft_body.cpp:1822-1929
 *   membrane_residual  updateMembraneSolverDiagnostics   soft_body.cpp:2366-2404
 *   material forms     complianceMatrix, effectiveMembraneStiffness,
 *                      checkedInverse (2x2, sym 3x3)     membrane.cpp:131-296
 *   payload_*          rigid payload                     suspension.cpp:1018-1102
 *   project_line       projectUnilateralLine             suspension.cpp:1104-1163
 *   begin_substep      SuspensionSystem::beginSubstep    suspension.cpp:2072-2182
 *   line_iteration     solveLineIteration                suspension.cpp:2197-2274
 *   certify/velocity/damping/finish                      suspension.cpp:2324-2610
 *   swo_diagnostics    Structure::diagnostics            structure.cpp:833-959
 *
 * Not restated (the functions return SWB_UNSUPPORTED): contact,
 * suspension controls and ground modes other than Free
 * (the Structure adapter always builds Free, structure.cpp:550), and the
 * equilibrated Cholesky fallback of a symmetric solve whose explicit inverse
 * is rejected (membrane.cpp:247-256).
 */
#include "simwing_b200.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double x, y, z; } V3;
typedef struct { double w, x, y, z; } Q;
typedef struct { double v[9]; } M3;

#ifdef SWO_FLOAT_VECTORS
/* The same algorithm with every vector result (positions, velocities, edges,
   normals, corrections) rounded to FP32 and the scalar arithmetic in FP64:
   the tests measure with it how strongly a configuration amplifies FP32
   rounding, which bounds what an FP32 solver can agree to. */
static V3 v3(double x, double y, double z) { V3 r = {(float)x, (float)y, (float)z}; return r; }
/* an FP32-rounded unit direction, checked as the FP32 device checks it */
static const double kUnitTolerance = 1.0e-5;
#else
static V3 v3(double x, double y, double z) { V3 r = {x, y, z}; return r; }
static const double kUnitTolerance = 1.0e-10; /* suspension.cpp:1140 */
#endif
static V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 mul(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 smul(double s, V3 a) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 vdiv(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
static V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z,
              a.x * b.y - a.y * b.x);
}
static double len(V3 a) { return sqrt(dot(a, a)); }
static V3 normalized(V3 a) {
    const double m = len(a);
    return m > 0.0 ? vdiv(a, m) : v3(0, 0, 0);
}
static int finite3(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
static int finiteq(Q q) {
    return isfinite(q.w) && isfinite(q.x) && isfinite(q.y) && isfinite(q.z);
}
static V3 fromabi(swb_vec3 a) { return v3(a.x, a.y, a.z); }
static swb_vec3 toabi(V3 a) { swb_vec3 r = {a.x, a.y, a.z}; return r; }

static const double kMinimumLength = 1.0e-12;       /* soft_body.cpp:38   */
static const double kFiniteTolerance = 1.0e-14;     /* suspension.cpp:27  */

static char g_error[512];
const char* swo_last_error(void) { return g_error; }
static swb_status fail(swb_status s, const char* message) {
    snprintf(g_error, sizeof g_error, "%s", message);
    return s;
}

/* ---------------- rigid payload helpers (suspension.cpp:538-690) -------- */
static double m3(const M3* m, int r, int c) { return m->v[r * 3 + c]; }
static M3 m3mul(const M3* a, const M3* b) {
    M3 r; memset(&r, 0, sizeof r);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k)
                r.v[i * 3 + j] += a->v[i * 3 + k] * b->v[k * 3 + j];
    return r;
}
static M3 m3t(const M3* a) {
    M3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.v[i * 3 + j] = a->v[j * 3 + i];
    return r;
}
static V3 m3v(const M3* m, V3 v) {
    return v3(m3(m, 0, 0) * v.x + m3(m, 0, 1) * v.y + m3(m, 0, 2) * v.z,
              m3(m, 1, 0) * v.x + m3(m, 1, 1) * v.y + m3(m, 1, 2) * v.z,
              m3(m, 2, 0) * v.x + m3(m, 2, 1) * v.y + m3(m, 2, 2) * v.z);
}
static double det3(const M3* m) {
    return m3(m, 0, 0) * (m3(m, 1, 1) * m3(m, 2, 2) - m3(m, 1, 2) * m3(m, 2, 1)) -
           m3(m, 0, 1) * (m3(m, 1, 0) * m3(m, 2, 2) - m3(m, 1, 2) * m3(m, 2, 0)) +
           m3(m, 0, 2) * (m3(m, 1, 0) * m3(m, 2, 1) - m3(m, 1, 1) * m3(m, 2, 0));
}
/* Mat3 inverse (suspension.cpp:567-595); returns 0 when singular. */
static int m3inv(const M3* m, M3* out) {
    double scale = 0.0;
    int best = 0;
    for (int i = 0; i < 9; ++i)
        if (fabs(m->v[i]) > fabs(m->v[best])) best = i;
    scale = fabs(m->v[best]);
    if (!(scale > 0.0) || !isfinite(scale)) return 0;
    M3 n = *m;
    for (int i = 0; i < 9; ++i) n.v[i] /= scale;
    const double det = det3(&n);
    if (!isfinite(det) || fabs(det) <= kFiniteTolerance) return 0;
    M3 r = {{
        m3(&n, 1, 1) * m3(&n, 2, 2) - m3(&n, 1, 2) * m3(&n, 2, 1),
        m3(&n, 0, 2) * m3(&n, 2, 1) - m3(&n, 0, 1) * m3(&n, 2, 2),
        m3(&n, 0, 1) * m3(&n, 1, 2) - m3(&n, 0, 2) * m3(&n, 1, 1),
        m3(&n, 1, 2) * m3(&n, 2, 0) - m3(&n, 1, 0) * m3(&n, 2, 2),
        m3(&n, 0, 0) * m3(&n, 2, 2) - m3(&n, 0, 2) * m3(&n, 2, 0),
        m3(&n, 0, 2) * m3(&n, 1, 0) - m3(&n, 0, 0) * m3(&n, 1, 2),
        m3(&n, 1, 0) * m3(&n, 2, 1) - m3(&n, 1, 1) * m3(&n, 2, 0),
        m3(&n, 0, 1) * m3(&n, 2, 0) - m3(&n, 0, 0) * m3(&n, 2, 1),
        m3(&n, 0, 0) * m3(&n, 1, 1) - m3(&n, 0, 1) * m3(&n, 1, 0)}};
    for (int i = 0; i < 9; ++i) r.v[i] /= det * scale;
    *out = r;
    return 1;
}
static double qnorm2(Q q) { return q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z; }
/* normalizedCanonical (suspension.cpp:617-636); returns 0 on failure. */
static int qcanon(Q q, Q* out) {
    const double n2 = qnorm2(q);
    if (!finiteq(q) || !(n2 > 1.0e-28)) return 0;
    const double inv = 1.0 / sqrt(n2);
    Q r = {q.w * inv, q.x * inv, q.y * inv, q.z * inv};
    const int flip = r.w < 0.0 ||
        (r.w == 0.0 && (r.x < 0.0 || (r.x == 0.0 && (r.y < 0.0 ||
                                                   (r.y == 0.0 && r.z < 0.0)))));
    if (flip) { r.w = -r.w; r.x = -r.x; r.y = -r.y; r.z = -r.z; }
    *out = r;
    return 1;
}
static Q qmul(Q a, Q b) {
    Q r = {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
           a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
           a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
           a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
    return r;
}
static int qrot(Q o, M3* out) {
    Q q;
    if (!qcanon(o, &q)) return 0;
    const double xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z;
    const double xy = q.x * q.y, xz = q.x * q.z, yz = q.y * q.z;
    const double wx = q.w * q.x, wy = q.w * q.y, wz = q.w * q.z;
    M3 r = {{1.0 - 2.0 * (yy + zz), 2.0 * (xy - wz), 2.0 * (xz + wy),
             2.0 * (xy + wz), 1.0 - 2.0 * (xx + zz), 2.0 * (yz - wx),
             2.0 * (xz - wy), 2.0 * (yz + wx), 1.0 - 2.0 * (xx + yy)}};
    *out = r;
    return 1;
}
/* rotationIncrement (suspension.cpp:669-684) */
static int qincrement(V3 r, Q* out) {
    if (!finite3(r)) return 0;
    const double angle = len(r);
    if (angle < 1.0e-12) {
        Q q = {1.0, 0.5 * r.x, 0.5 * r.y, 0.5 * r.z};
        return qcanon(q, out);
    }
    const double half = 0.5 * angle;
    const double scale = sin(half) / angle;
    Q q = {cos(half), r.x * scale, r.y * scale, r.z * scale};
    *out = q;
    return 1;
}

typedef struct {
    double mass;
    V3 com_local;
    M3 inertia_body;
} PayloadDef;
typedef struct {
    V3 com;
    Q orientation;
    V3 linear_velocity;
    V3 angular_velocity;
} Payload;

static int world_inertia(const PayloadDef* d, const Payload* s, M3* out) {
    M3 r;
    if (!qrot(s->orientation, &r)) return 0;
    M3 t = m3t(&r);
    M3 a = m3mul(&r, &d->inertia_body);
    *out = m3mul(&a, &t);
    return 1;
}
static int point_position(const PayloadDef* d, const Payload* s, V3 local, V3* out) {
    M3 r;
    if (!qrot(s->orientation, &r)) return 0;
    *out = add(s->com, m3v(&r, sub(local, d->com_local)));
    return 1;
}
static int point_velocity(const PayloadDef* d, const Payload* s, V3 local, V3* out) {
    M3 r;
    if (!qrot(s->orientation, &r)) return 0;
    const V3 offset = m3v(&r, sub(local, d->com_local));
    *out = add(s->linear_velocity, cross(s->angular_velocity, offset));
    return 1;
}
/* integratePayloadTorqueFree (suspension.cpp:1075-1102) */
static int integrate_payload(const PayloadDef* d, Payload* s, double dt,
                             V3 force, V3 moment) {
    if (!(dt > 0.0) || !isfinite(dt) || !finite3(force) || !finite3(moment))
        return 0;
    if (!qcanon(s->orientation, &s->orientation)) return 0;
    M3 inertia, inv;
    if (!world_inertia(d, s, &inertia)) return 0;
    V3 angular = m3v(&inertia, s->angular_velocity);
    s->linear_velocity = add(s->linear_velocity, mul(force, dt / d->mass));
    angular = add(angular, mul(moment, dt));
    if (!m3inv(&inertia, &inv)) return 0;
    s->angular_velocity = m3v(&inv, angular);
    s->com = add(s->com, mul(s->linear_velocity, dt));
    Q inc;
    if (!qincrement(mul(s->angular_velocity, dt), &inc)) return 0;
    if (!qcanon(qmul(inc, s->orientation), &s->orientation)) return 0;
    if (!world_inertia(d, s, &inertia) || !m3inv(&inertia, &inv)) return 0;
    s->angular_velocity = m3v(&inv, angular);
    return finite3(s->com) && finite3(s->linear_velocity) &&
           finite3(s->angular_velocity) && finiteq(s->orientation);
}

/* ---------------- model --------------------------------------------------- */
typedef struct {
    V3 x, prev, v, force;
    double w;
} Node;
typedef struct {
    uint64_t a, b;
    double rest, compliance, lambda;
    uint32_t kind;
} Distance;
typedef struct {
    uint64_t a, b, c, d;
    double rest, compliance, lambda;
} Dihedral;
typedef struct { double xx, yy, zz, xy, xz, yz; } S3;
typedef struct {
    uint64_t a, b, c;                /* the element's triangle corners      */
    double inv00, inv01, inv10, inv11; /* inverse reference (chart) matrix  */
    double area;                     /* reference area                      */
    S3 stiffness, compliance;        /* material stiffness and its inverse  */
    double warp_pre, weft_pre, damping_time, compression_ratio;
    V3 multiplier;
    double residual;                 /* normalizedResidual of the last substep */
} Membrane;
typedef struct {
    int from_node, to_node;      /* node index or -1                     */
    int from_point, to_point;    /* hang-point index or -1               */
    double rest, stiffness, damping, lambda, commanded;
    uint64_t stable_id;
    uint64_t definition_index;
} Segment;

typedef struct swo_structure {
    uint64_t n, t, m, h, nm;
    Membrane* mem;
    uint64_t* load_path;     /* cable and tie indices in load-path order  */
    uint64_t nload;
    Node* nodes;
    uint64_t (*tri)[3];
    double* pressure;
    Distance* dist;
    Dihedral* dih;
    V3* pending;
    V3 last_applied;
    uint64_t accepted;
    double time;
    /* suspension */
    int has_suspension;
    PayloadDef pdef;
    Payload payload, previous_payload;
    uint64_t nseg, nhang;
    Segment* seg;
    V3* hang_local;          /* sorted by id like the reference          */
    int line_iterations;
    double minimum_line_length, maximum_line_residual;
    double max_residual;
    V3 line_force, line_moment;
    /* ground plane (swb_structure_set_ground; no counterpart in the
     * reference, so its parity is the device's against this restatement) */
    int ground;
    V3 ground_normal;
    double ground_offset, ground_friction;
    /* line-line contact (swb_structure_set_line_contact; the reference
     * rejects segment contact, so its parity is the device's against this
     * restatement): cable segments by (smaller, larger) node, the substep's
     * candidate pairs in key order */
    int lines;
    double line_radius, line_reach;
    uint64_t nseg_lines, npairs, pairs_cap;
    uint64_t (*line_seg)[2];
    uint64_t (*line_pair)[2];
} swo_structure;

/* ---------------- membranes (soft_body.cpp, membrane.cpp) ---------------- */
static const double kEpsilon = 2.220446049250313080847e-16;

/* checkedInverse(Matrix2) (membrane.cpp:131-151): m = {m00, m01, m10, m11} */
static int inverse2(const double m[4], double out[4]) {
    for (int i = 0; i < 4; ++i)
        if (!isfinite(m[i])) return 0;
    double scale = fabs(m[0]);
    for (int i = 1; i < 4; ++i) scale = fabs(m[i]) > scale ? fabs(m[i]) : scale;
    const double det = m[0] * m[3] - m[1] * m[2];
    const double tol = 64.0 * kEpsilon * scale * scale;
    if (!(scale > 0.0) || !isfinite(det) || fabs(det) <= tol) return 0;
    const double id = 1.0 / det;
    out[0] = m[3] * id; out[1] = -m[1] * id; out[2] = -m[2] * id; out[3] = m[0] * id;
    return 1;
}
/* checkedInverse(SymmetricMatrix3) (membrane.cpp:208-235) */
static int inverse_s3(const S3* m, S3* out) {
    const double e[6] = {m->xx, m->yy, m->zz, m->xy, m->xz, m->yz};
    double scale = 0.0;
    for (int i = 0; i < 6; ++i) {
        if (!isfinite(e[i])) return 0;
        scale = fabs(e[i]) > scale ? fabs(e[i]) : scale;
    }
    const double det = m->xx * (m->yy * m->zz - m->yz * m->yz) -
                       m->xy * (m->xy * m->zz - m->yz * m->xz) +
                       m->xz * (m->xy * m->yz - m->yy * m->xz);
    const double tol = 128.0 * kEpsilon * scale * scale * scale;
    if (!(scale > 0.0) || !isfinite(det) || fabs(det) <= tol) return 0;
    const double id = 1.0 / det;
    out->xx = (m->yy * m->zz - m->yz * m->yz) * id;
    out->yy = (m->xx * m->zz - m->xz * m->xz) * id;
    out->zz = (m->xx * m->yy - m->xy * m->xy) * id;
    out->xy = (m->xz * m->yz - m->xy * m->zz) * id;
    out->xz = (m->xy * m->yz - m->xz * m->yy) * id;
    out->yz = (m->xy * m->xz - m->xx * m->yz) * id;
    return 1;
}
static V3 s3v(const S3* m, V3 v) {
    return v3(m->xx * v.x + m->xy * v.y + m->xz * v.z,
              m->xy * v.x + m->yy * v.y + m->yz * v.z,
              m->xz * v.x + m->yz * v.y + m->zz * v.z);
}
static S3 s3scale(double s, const S3* m) {
    S3 r = {s * m->xx, s * m->yy, s * m->zz, s * m->xy, s * m->xz, s * m->yz};
    return r;
}
static S3 s3add(const S3* a, const S3* b) {
    S3 r = {a->xx + b->xx, a->yy + b->yy, a->zz + b->zz, a->xy + b->xy, a->xz + b->xz, a->yz + b->yz};
    return r;
}

/* addMembraneElements (soft_body.cpp:664-690) with the material's
 * stiffnessMatrix / complianceMatrix (membrane.cpp:259-271) */
static int membrane_setup(const swb_membrane_def* d, const swb_triangle_def* tris, Membrane* e) {
    const swb_triangle_def* t = &tris[d->triangle];
    e->a = t->nodes[0]; e->b = t->nodes[1]; e->c = t->nodes[2];
    const double e1x = d->chart[1][0] - d->chart[0][0], e1y = d->chart[1][1] - d->chart[0][1];
    const double e2x = d->chart[2][0] - d->chart[0][0], e2y = d->chart[2][1] - d->chart[0][1];
    const double ref[4] = {e1x, e2x, e1y, e2y};
    double inv[4];
    e->area = 0.5 * (ref[0] * ref[3] - ref[1] * ref[2]);
    if (!inverse2(ref, inv)) return 0;
    e->inv00 = inv[0]; e->inv01 = inv[1]; e->inv10 = inv[2]; e->inv11 = inv[3];
    const swb_membrane_material* m = &d->material;
    S3 k = {m->warp_stiffness, m->weft_stiffness, m->shear_stiffness, m->coupling_stiffness, 0.0, 0.0};
    e->stiffness = k;
    if (!inverse_s3(&k, &e->compliance)) return 0;
    e->warp_pre = m->warp_pretension;
    e->weft_pre = m->weft_pretension;
    e->damping_time = m->damping_seconds;
    e->compression_ratio = m->compression_stiffness_ratio;
    return 1;
}

/* effectiveMembraneStiffness (membrane.cpp:273-296) */
static S3 effective_stiffness(const Membrane* e, V3 strain) {
    if (e->compression_ratio == 1.0) return e->stiffness;
    const double retained = sqrt(e->compression_ratio);
    const double ws = strain.x < 0.0 ? retained : 1.0;
    const double fs = strain.y < 0.0 ? retained : 1.0;
    const double ss = sqrt(ws * fs);
    const S3* k = &e->stiffness;
    S3 r = {k->xx * ws * ws, k->yy * fs * fs, k->zz * ss * ss, k->xy * ws * fs, k->xz * ws * ss, k->yz * fs * ss};
    return r;
}

/* evaluateMembraneElement, strain and its gradients (soft_body.cpp:204-270):
 * g[component][corner] */
static V3 membrane_strain(const Node* nodes, const Membrane* e, V3 g[3][3]) {
    const V3 pa = nodes[e->a].x, pb = nodes[e->b].x, pc = nodes[e->c].x;
    const V3 e1 = sub(pb, pa), e2 = sub(pc, pa);
    const V3 warp = add(smul(e->inv00, e1), smul(e->inv10, e2));
    const V3 weft = add(smul(e->inv01, e1), smul(e->inv11, e2));
    const V3 strain = v3(0.5 * (dot(warp, warp) - 1.0) + e->warp_pre,
                         0.5 * (dot(weft, weft) - 1.0) + e->weft_pre, dot(warp, weft));
    const V3 zero = v3(0, 0, 0);
    const V3 by_warp[3] = {warp, zero, weft};
    const V3 by_weft[3] = {zero, weft, warp};
    for (int c = 0; c < 3; ++c) {
        const V3 first = add(smul(e->inv00, by_warp[c]), smul(e->inv01, by_weft[c]));
        const V3 second = add(smul(e->inv10, by_warp[c]), smul(e->inv11, by_weft[c]));
        g[c][0] = neg(add(first, second));
        g[c][1] = first;
        g[c][2] = second;
    }
    return strain;
}

static int checked_solve(const S3* m, V3 rhs, V3* out);

/* membraneElementCorrections + solveMembraneElement (soft_body.cpp:1822-1929) */
static int solve_membrane(swo_structure* s, Membrane* e, double dt) {
    V3 g[3][3];
    const V3 strain = membrane_strain(s->nodes, e, g);
    const uint64_t idx[3] = {e->a, e->b, e->c};
    const double area_scale = sqrt(e->area);
    V3 J[3][3];
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) J[c][k] = mul(g[c][k], area_scale);
    S3 M = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        const double w = s->nodes[idx[k]].w;
        M.xx += w * dot(J[0][k], J[0][k]);
        M.yy += w * dot(J[1][k], J[1][k]);
        M.zz += w * dot(J[2][k], J[2][k]);
        M.xy += w * dot(J[0][k], J[1][k]);
        M.xz += w * dot(J[0][k], J[2][k]);
        M.yz += w * dot(J[1][k], J[2][k]);
    }
    V3 damping = v3(0, 0, 0);
    for (int k = 0; k < 3; ++k) {
        const V3 disp = sub(s->nodes[idx[k]].x, s->nodes[idx[k]].prev);
        damping.x += dot(J[0][k], disp);
        damping.y += dot(J[1][k], disp);
        damping.z += dot(J[2][k], disp);
    }
    const double inv_dt2 = 1.0 / (dt * dt);
    S3 compliance = e->compliance;
    if (!(e->compression_ratio == 1.0)) {
        const S3 k = effective_stiffness(e, strain);
        if (!inverse_s3(&k, &compliance)) return 0;
    }
    const S3 alpha = s3scale(inv_dt2, &compliance);
    const double gamma = e->damping_time / dt;
    const S3 Ms = s3scale(1.0 + gamma, &M);
    const S3 system = s3add(&Ms, &alpha);
    const V3 value = smul(area_scale, strain);
    const V3 rhs = sub(sub(neg(value), s3v(&alpha, e->multiplier)), smul(gamma, damping));
    if (!finite3(rhs)) return 0;
    V3 dl;
    if (!checked_solve(&system, rhs, &dl)) return 0;
    V3 corr[3];
    for (int k = 0; k < 3; ++k) {
        const V3 c = add(add(mul(J[0][k], dl.x), mul(J[1][k], dl.y)), mul(J[2][k], dl.z));
        corr[k] = smul(s->nodes[idx[k]].w, c);
    }
    e->multiplier = add(e->multiplier, dl);
    for (int k = 0; k < 3; ++k) s->nodes[idx[k]].x = add(s->nodes[idx[k]].x, corr[k]);
    return 1;
}

/* updateMembraneSolverDiagnostics: the normalized residual (soft_body.cpp:2366-2404) */
static void membrane_residual(swo_structure* s, Membrane* e, double dt) {
    V3 g[3][3];
    const V3 strain = membrane_strain(s->nodes, e, g);
    const uint64_t idx[3] = {e->a, e->b, e->c};
    const double area_scale = sqrt(e->area);
    const double inv_dt2 = 1.0 / (dt * dt);
    const S3 alpha = s3scale(inv_dt2, &e->compliance);
    const double gamma = e->damping_time / dt;
    V3 damping = v3(0, 0, 0);
    for (int k = 0; k < 3; ++k) {
        const V3 disp = sub(s->nodes[idx[k]].x, s->nodes[idx[k]].prev);
        damping.x += area_scale * dot(g[0][k], disp);
        damping.y += area_scale * dot(g[1][k], disp);
        damping.z += area_scale * dot(g[2][k], disp);
    }
    const V3 r = add(add(smul(area_scale, strain), s3v(&alpha, e->multiplier)), smul(gamma, damping));
    e->residual = len(r) / area_scale;
}

static int cmp_u64str(uint64_t a, uint64_t b) {
    char sa[32], sb[32];
    snprintf(sa, sizeof sa, "%llu", (unsigned long long)a);
    snprintf(sb, sizeof sb, "%llu", (unsigned long long)b);
    return strcmp(sa, sb);
}

/* loadPathConstraintOrder (soft_body.cpp:528-629): the cables and
 * suspension ties, stable-sorted by graph depth from the structural skin
 * (fixed nodes and every node of a triangle, distance or seam constraint, or
 * dihedral); a component with no structural node is rooted at its heaviest
 * node (the first of the smallest inverse mass). */
static void load_path_order(swo_structure* s) {
    const uint64_t n = s->n;
    uint8_t* structural = calloc(n ? n : 1, 1);
    uint64_t* deg = calloc(n + 1, sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) structural[i] = s->nodes[i].w == 0.0;
    for (uint64_t t = 0; t < s->t; ++t)
        for (int k = 0; k < 3; ++k) structural[s->tri[t][k]] = 1;
    s->nload = 0;
    for (uint64_t i = 0; i < s->m; ++i) {
        const Distance* c = &s->dist[i];
        if (c->kind == SWB_CONSTRAINT_DISTANCE || c->kind == SWB_CONSTRAINT_SEAM_STITCH) {
            structural[c->a] = structural[c->b] = 1;
            continue;
        }
        ++s->nload;
        ++deg[c->a + 1];
        ++deg[c->b + 1];
    }
    for (uint64_t i = 0; i < s->h; ++i) {
        structural[s->dih[i].a] = structural[s->dih[i].b] = 1;
        structural[s->dih[i].c] = structural[s->dih[i].d] = 1;
    }
    for (uint64_t v = 0; v < n; ++v) deg[v + 1] += deg[v];
    /* adjacency in constraint order (each node's neighbours in the order
     * its load-path constraints appear) */
    uint64_t* adj = malloc((2 * s->nload + 1) * sizeof(uint64_t));
    uint64_t* cur = malloc((n + 1) * sizeof(uint64_t));
    memcpy(cur, deg, (n + 1) * sizeof(uint64_t));
    free(s->load_path);
    s->load_path = malloc((s->nload + 1) * sizeof(uint64_t));
    uint64_t k = 0;
    for (uint64_t i = 0; i < s->m; ++i) {
        const Distance* c = &s->dist[i];
        if (c->kind == SWB_CONSTRAINT_DISTANCE || c->kind == SWB_CONSTRAINT_SEAM_STITCH) continue;
        s->load_path[k++] = i;
        adj[cur[c->a]++] = c->b;
        adj[cur[c->b]++] = c->a;
    }
    const uint64_t unknown = ~(uint64_t)0;
    uint64_t* depth = malloc((n ? n : 1) * sizeof(uint64_t));
    uint64_t* queue = malloc((n ? n : 1) * sizeof(uint64_t));
    uint64_t head = 0, tail = 0;
    for (uint64_t v = 0; v < n; ++v) {
        depth[v] = unknown;
        if (structural[v] && deg[v + 1] > deg[v]) {
            depth[v] = 0;
            queue[tail++] = v;
        }
    }
    for (;;) {
        while (head < tail) {
            const uint64_t v = queue[head++];
            for (uint64_t e = deg[v]; e < deg[v + 1]; ++e)
                if (depth[adj[e]] == unknown) {
                    depth[adj[e]] = depth[v] + 1;
                    queue[tail++] = adj[e];
                }
        }
        uint64_t root = n;
        double smallest = INFINITY;
        for (uint64_t v = 0; v < n; ++v)
            if (depth[v] == unknown && deg[v + 1] > deg[v] && s->nodes[v].w < smallest) {
                root = v;
                smallest = s->nodes[v].w;
            }
        if (root == n) break;
        depth[root] = 0;
        queue[tail++] = root;
    }
    /* stable insertion sort by max(depth[a], depth[b]) */
    for (uint64_t i = 1; i < s->nload; ++i) {
        const uint64_t x = s->load_path[i];
        const uint64_t dx = depth[s->dist[x].a] > depth[s->dist[x].b] ? depth[s->dist[x].a] : depth[s->dist[x].b];
        uint64_t j = i;
        while (j > 0) {
            const uint64_t y = s->load_path[j - 1];
            const uint64_t dy = depth[s->dist[y].a] > depth[s->dist[y].b] ? depth[s->dist[y].a] : depth[s->dist[y].b];
            if (dy <= dx) break;
            s->load_path[j] = y;
            --j;
        }
        s->load_path[j] = x;
    }
    free(structural); free(deg); free(adj); free(cur); free(depth); free(queue);
}

static void project_distance(swo_structure* s, Distance* c, double inv_dt2);

/* solveCablePair (soft_body.cpp:1265-1286): reverse depth order, then
 * forward depth order */
static void cable_pair(swo_structure* s, double inv_dt2) {
    for (uint64_t k = s->nload; k-- > 0;) project_distance(s, &s->dist[s->load_path[k]], inv_dt2);
    for (uint64_t k = 0; k < s->nload; ++k) project_distance(s, &s->dist[s->load_path[k]], inv_dt2);
}

void swo_destroy(swo_structure* s) {
    if (!s) return;
    free(s->nodes); free(s->tri); free(s->pressure); free(s->dist);
    free(s->dih); free(s->pending); free(s->seg); free(s->hang_local); free(s->mem); free(s->load_path);
    free(s->line_seg); free(s->line_pair);
    free(s);
}

swb_status swo_create(const swb_structure_definition* d, swo_structure** out) {
    if (d->fabric_self_contact)
        return fail(SWB_UNSUPPORTED, "oracle port: contact not restated");
    swo_structure* s = calloc(1, sizeof *s);
    s->n = d->node_count; s->t = d->triangle_count;
    s->m = d->constraint_count; s->h = d->dihedral_count;
    s->nodes = calloc(s->n ? s->n : 1, sizeof(Node));
    s->pending = calloc(s->n ? s->n : 1, sizeof(V3));
    s->tri = calloc(s->t ? s->t : 1, sizeof *s->tri);
    s->pressure = calloc(s->t ? s->t : 1, sizeof(double));
    s->dist = calloc(s->m ? s->m : 1, sizeof(Distance));
    s->dih = calloc(s->h ? s->h : 1, sizeof(Dihedral));
    for (uint64_t i = 0; i < s->n; ++i) {
        const swb_node_def* nd = &d->nodes[i];
        s->nodes[i].x = fromabi(nd->position);
        s->nodes[i].prev = s->nodes[i].x;
        /* addNode: inverse mass 1/m; addFixedNode: 0 (soft_body.cpp) */
        s->nodes[i].w = nd->fixed ? 0.0 : 1.0 / nd->mass;
    }
    for (uint64_t i = 0; i < s->t; ++i) {
        for (int k = 0; k < 3; ++k) s->tri[i][k] = d->triangles[i].nodes[k];
        s->pressure[i] = d->triangles[i].pressure_difference;
    }
    for (uint64_t i = 0; i < s->m; ++i) {
        const swb_constraint_def* c = &d->constraints[i];
        s->dist[i].a = c->first_node;
        s->dist[i].b = c->second_node;
        s->dist[i].kind = c->kind;
        s->dist[i].rest = c->kind == SWB_CONSTRAINT_SEAM_STITCH ? 0.0 : c->rest_length;
        s->dist[i].compliance =
            c->kind == SWB_CONSTRAINT_SEAM_STITCH ? 0.0 : c->compliance;
    }
    load_path_order(s);
    s->nm = d->membrane_count;
    s->mem = calloc(s->nm ? s->nm : 1, sizeof(Membrane));
    for (uint64_t i = 0; i < s->nm; ++i)
        if (!membrane_setup(&d->membranes[i], d->triangles, &s->mem[i])) {
            swo_destroy(s);
            return fail(SWB_INVALID_ARGUMENT, "membrane chart or material is singular");
        }
    for (uint64_t i = 0; i < s->h; ++i) {
        const swb_dihedral_def* h = &d->dihedrals[i];
        s->dih[i].a = h->nodes[0]; s->dih[i].b = h->nodes[1];
        s->dih[i].c = h->nodes[2]; s->dih[i].d = h->nodes[3];
        s->dih[i].rest = h->rest_angle;
        s->dih[i].compliance = h->compliance;
    }
    if (d->suspension) {
        const swb_suspension_def* sp = d->suspension;
        s->has_suspension = 1;
        s->pdef.mass = sp->pilot_mass;
        s->pdef.com_local = fromabi(sp->pilot_com_local);
        memset(&s->pdef.inertia_body, 0, sizeof(M3));
        s->pdef.inertia_body.v[0] = sp->pilot_principal_inertia.x;
        s->pdef.inertia_body.v[4] = sp->pilot_principal_inertia.y;
        s->pdef.inertia_body.v[8] = sp->pilot_principal_inertia.z;
        s->payload.com = fromabi(sp->pilot_initial_com_world);
        s->payload.orientation.w = sp->pilot_initial_body_to_world.w;
        s->payload.orientation.x = sp->pilot_initial_body_to_world.x;
        s->payload.orientation.y = sp->pilot_initial_body_to_world.y;
        s->payload.orientation.z = sp->pilot_initial_body_to_world.z;
        /* validateAndNormalizeSuspensionDefinition canonicalises the
         * initial orientation (suspension.cpp:771). */
        if (!qcanon(s->payload.orientation, &s->payload.orientation)) {
            swo_destroy(s);
            return fail(SWB_SUSPENSION_ERROR, "invalid pilot orientation");
        }
        s->payload.linear_velocity = fromabi(sp->pilot_initial_linear_velocity);
        s->payload.angular_velocity = fromabi(sp->pilot_initial_angular_velocity);
        s->previous_payload = s->payload;
        s->line_iterations = sp->solver_iterations;
        s->minimum_line_length = sp->minimum_line_length;
        s->maximum_line_residual = sp->maximum_line_residual;
        /* Hang points and segments are sorted by their string ids
         * "harness:<id>" / "segment:<id>" (suspension.cpp:1000-1006). */
        s->nhang = sp->harness_count;
        s->hang_local = calloc(s->nhang ? s->nhang : 1, sizeof(V3));
        uint64_t* hang_order = calloc(s->nhang ? s->nhang : 1, sizeof(uint64_t));
        for (uint64_t i = 0; i < s->nhang; ++i) hang_order[i] = i;
        for (uint64_t i = 1; i < s->nhang; ++i)
            for (uint64_t j = i; j > 0 &&
                 cmp_u64str(sp->harness_points[hang_order[j]].stable_id,
                            sp->harness_points[hang_order[j - 1]].stable_id) < 0; --j) {
                uint64_t tmp = hang_order[j]; hang_order[j] = hang_order[j - 1];
                hang_order[j - 1] = tmp;
            }
        for (uint64_t i = 0; i < s->nhang; ++i)
            s->hang_local[i] = fromabi(sp->harness_points[hang_order[i]].local_position);
        s->nseg = sp->segment_count;
        s->seg = calloc(s->nseg ? s->nseg : 1, sizeof(Segment));
        uint64_t* order = calloc(s->nseg ? s->nseg : 1, sizeof(uint64_t));
        for (uint64_t i = 0; i < s->nseg; ++i) order[i] = i;
        for (uint64_t i = 1; i < s->nseg; ++i)
            for (uint64_t j = i; j > 0 &&
                 cmp_u64str(sp->segments[order[j]].stable_id,
                            sp->segments[order[j - 1]].stable_id) < 0; --j) {
                uint64_t tmp = order[j]; order[j] = order[j - 1]; order[j - 1] = tmp;
            }
        for (uint64_t k = 0; k < s->nseg; ++k) {
            const swb_suspension_segment* g = &sp->segments[order[k]];
            Segment* r = &s->seg[k];
            r->definition_index = order[k];
            r->stable_id = g->stable_id;
            r->rest = g->rest_length;
            r->commanded = g->rest_length;
            r->stiffness = g->axial_stiffness;
            r->damping = g->axial_damping;
            r->from_node = r->to_node = r->from_point = r->to_point = -1;
            const swb_suspension_endpoint* ends[2] = {&g->from, &g->to};
            for (int e = 0; e < 2; ++e) {
                int node = -1, point = -1;
                if (ends[e]->kind == SWB_ENDPOINT_SURFACE_ATTACHMENT) {
                    for (uint64_t a = 0; a < sp->attachment_count; ++a)
                        if (sp->attachments[a].stable_id == ends[e]->stable_id)
                            node = (int)sp->attachments[a].node;
                } else if (ends[e]->kind == SWB_ENDPOINT_JUNCTION) {
                    for (uint64_t a = 0; a < sp->junction_count; ++a)
                        if (sp->junctions[a].stable_id == ends[e]->stable_id)
                            node = (int)sp->junctions[a].node;
                } else {
                    for (uint64_t a = 0; a < s->nhang; ++a)
                        if (sp->harness_points[hang_order[a]].stable_id ==
                            ends[e]->stable_id)
                            point = (int)a;
                }
                if (e == 0) { r->from_node = node; r->from_point = point; }
                else { r->to_node = node; r->to_point = point; }
            }
        }
        free(order);
        free(hang_order);
    }
    *out = s;
    return SWB_OK;
}

swb_status swo_set_external_forces(swo_structure* s, const swb_vec3* f, uint64_t n) {
    if (n != s->n) return fail(SWB_INVALID_ARGUMENT, "force count must equal node count");
    for (uint64_t i = 0; i < n; ++i) {
        if (!finite3(fromabi(f[i]))) return fail(SWB_INVALID_ARGUMENT, "non-finite force");
    }
    for (uint64_t i = 0; i < n; ++i) s->pending[i] = fromabi(f[i]);
    return SWB_OK;
}

swb_status swo_add_external_force(swo_structure* s, uint64_t node, const swb_vec3* f) {
    if (node >= s->n) return fail(SWB_OUT_OF_RANGE, "node out of range");
    if (!finite3(fromabi(*f))) return fail(SWB_INVALID_ARGUMENT, "non-finite force");
    s->pending[node] = add(s->pending[node], fromabi(*f));
    return SWB_OK;
}

/* ---------------- soft body kernels -------------------------------------- */
static void pressure_scatter(swo_structure* s) {
    for (uint64_t t = 0; t < s->t; ++t) {
        const V3 a = s->nodes[s->tri[t][0]].x;
        const V3 b = s->nodes[s->tri[t][1]].x;
        const V3 c = s->nodes[s->tri[t][2]].x;
        const V3 area = smul(0.5, cross(sub(b, a), sub(c, a)));
        const V3 f = vdiv(smul(s->pressure[t], area), 3.0);
        for (int k = 0; k < 3; ++k)
            s->nodes[s->tri[t][k]].force = add(s->nodes[s->tri[t][k]].force, f);
    }
}

static void predict(swo_structure* s, double dt, V3 g, double damping, V3 ref) {
    for (uint64_t i = 0; i < s->n; ++i) {
        Node* n = &s->nodes[i];
        n->prev = n->x;
        if (n->w == 0.0) { n->v = v3(0, 0, 0); continue; }
        const V3 acc = add(g, mul(n->force, n->w));
        n->v = add(ref, mul(sub(add(n->v, mul(acc, dt)), ref), damping));
        n->x = add(n->x, mul(n->v, dt));
    }
}

static void finalize(swo_structure* s, double dt) {
    const double inv = 1.0 / dt;
    for (uint64_t i = 0; i < s->n; ++i) {
        Node* n = &s->nodes[i];
        n->v = n->w == 0.0 ? v3(0, 0, 0) : mul(sub(n->x, n->prev), inv);
    }
}

static void project_distance(swo_structure* s, Distance* c, double inv_dt2) {
    Node* na = &s->nodes[c->a];
    Node* nb = &s->nodes[c->b];
    const V3 diff = sub(nb->x, na->x);
    const double l = len(diff);
    if (l <= kMinimumLength) return;
    const double value = l - c->rest;
    if (c->kind == SWB_CONSTRAINT_CABLE && value <= 0.0 && c->lambda == 0.0) return;
    const double wsum = na->w + nb->w;
    const double alpha = c->compliance * inv_dt2;
    if (wsum + alpha <= 0.0) return;
    const double dl = (-value - alpha * c->lambda) / (wsum + alpha);
    double applied = dl;
    if (c->kind == SWB_CONSTRAINT_CABLE) {
        const double nl = fmin(0.0, c->lambda + dl);
        /* std::min(0.0, x) returns 0.0 unless x < 0.0 */
        const double newl = (c->lambda + dl) < 0.0 ? (c->lambda + dl) : 0.0;
        (void)nl;
        applied = newl - c->lambda;
        c->lambda = newl;
    } else {
        c->lambda += dl;
    }
    const double scale = applied / l;
    na->x = sub(na->x, mul(diff, na->w * scale));
    nb->x = add(nb->x, mul(diff, nb->w * scale));
}

typedef struct { double angle; V3 g[4]; int valid; } DihedralEval;

static DihedralEval evaluate_dihedral(V3 a, V3 b, V3 c, V3 d) {
    DihedralEval r; memset(&r, 0, sizeof r);
    const V3 edge = sub(b, a);
    const V3 toC = sub(c, a);
    const V3 toD = sub(d, a);
    const V3 A1 = cross(edge, toC);
    const V3 A2 = cross(toD, edge);
    const double el = len(edge), l1 = len(A1), l2 = len(A2);
    if (!(el > kMinimumLength) || !(l1 > kMinimumLength * el) ||
        !(l2 > kMinimumLength * el))
        return r;
    const V3 e = vdiv(edge, el);
    const V3 n1 = vdiv(A1, l1);
    const V3 n2 = vdiv(A2, l2);
    double cosine = dot(n1, n2);
    cosine = cosine < -1.0 ? -1.0 : (1.0 < cosine ? 1.0 : cosine);
    const double sine = dot(e, cross(n1, n2));
    const V3 n1adj = sub(smul(cosine, cross(n2, e)), smul(sine, n2));
    const V3 n2adj = sub(smul(cosine, cross(e, n1)), smul(sine, n1));
    const V3 eadj = smul(cosine, cross(n1, n2));
    const V3 a1adj = vdiv(sub(n1adj, smul(dot(n1adj, n1), n1)), l1);
    const V3 a2adj = vdiv(sub(n2adj, smul(dot(n2adj, n2), n2)), l2);
    V3 edgeadj = vdiv(sub(eadj, smul(dot(eadj, e), e)), el);
    edgeadj = add(edgeadj, cross(toC, a1adj));
    const V3 cadj = cross(a1adj, edge);
    edgeadj = add(edgeadj, cross(a2adj, toD));
    const V3 dadj = cross(edge, a2adj);
    r.angle = atan2(sine, cosine);
    r.g[1] = edgeadj;
    r.g[2] = cadj;
    r.g[3] = dadj;
    r.g[0] = smul(-1.0, add(add(edgeadj, cadj), dadj));
    r.valid = isfinite(r.angle) && finite3(r.g[0]) && finite3(r.g[1]) &&
              finite3(r.g[2]) && finite3(r.g[3]);
    return r;
}

static void solve_dihedral(swo_structure* s, Dihedral* c, double inv_dt2) {
    const uint64_t idx[4] = {c->a, c->b, c->c, c->d};
    const DihedralEval ev = evaluate_dihedral(s->nodes[c->a].x, s->nodes[c->b].x,
                                              s->nodes[c->c].x, s->nodes[c->d].x);
    if (!ev.valid) return;
    double wg = 0.0;
    for (int k = 0; k < 4; ++k) wg += s->nodes[idx[k]].w * dot(ev.g[k], ev.g[k]);
    const double alpha = c->compliance * inv_dt2;
    const double den = wg + alpha;
    if (!(den > 0.0) || !isfinite(den)) return;
    const double twoPi = 6.283185307179586476925286766559;
    const double value = remainder(ev.angle - c->rest, twoPi);
    const double dl = (-value - alpha * c->lambda) / den;
    if (!isfinite(dl)) return;
    for (int k = 0; k < 4; ++k) {
        Node* n = &s->nodes[idx[k]];
        n->x = add(n->x, smul(n->w * dl, ev.g[k]));
    }
    c->lambda += dl;
}

/* ---------------- momentum guard (soft_body.cpp:119-190) ----------------- */
typedef struct { double mass; V3 com, p, L; } Momentum;
static Momentum measure_momentum(const swo_structure* s) {
    Momentum r; memset(&r, 0, sizeof r);
    for (uint64_t i = 0; i < s->n; ++i) {
        const Node* n = &s->nodes[i];
        if (n->w <= 0.0) continue;
        const double m = 1.0 / n->w;
        r.mass += m;
        r.com = add(r.com, smul(m, n->x));
        r.p = add(r.p, smul(m, n->v));
    }
    if (!(r.mass > 0.0)) return r;
    r.com = vdiv(r.com, r.mass);
    for (uint64_t i = 0; i < s->n; ++i) {
        const Node* n = &s->nodes[i];
        if (n->w <= 0.0) continue;
        const double m = 1.0 / n->w;
        r.L = add(r.L, smul(m, cross(sub(n->x, r.com), n->v)));
    }
    return r;
}
static int spd(const S3* m) {
    if (!isfinite(m->xx) || !isfinite(m->yy) || !isfinite(m->zz) ||
        !isfinite(m->xy) || !isfinite(m->xz) || !isfinite(m->yz) ||
        !(m->xx > 0.0) || !(m->yy > 0.0) || !(m->zz > 0.0))
        return 0;
    const double sx = sqrt(m->xx), sy = sqrt(m->yy), sz = sqrt(m->zz);
    const double l10 = m->xy / sx / sy;
    const double l20 = m->xz / sx / sz;
    const double p1 = 1.0 - l10 * l10;
    if (!isfinite(p1) || !(p1 > 0.0)) return 0;
    const double l11 = sqrt(p1);
    const double l21 = (m->yz / sy / sz - l20 * l10) / l11;
    const double p2 = 1.0 - l20 * l20 - l21 * l21;
    return isfinite(p2) && p2 > 0.0;
}
static int checked_solve(const S3* m, V3 rhs, V3* out) {
    double scale = fabs(m->xx);
    const double e[5] = {m->yy, m->zz, m->xy, m->xz, m->yz};
    for (int i = 0; i < 5; ++i) if (fabs(e[i]) > scale) scale = fabs(e[i]);
    const double det = m->xx * (m->yy * m->zz - m->yz * m->yz) -
                       m->xy * (m->xy * m->zz - m->yz * m->xz) +
                       m->xz * (m->xy * m->yz - m->yy * m->xz);
    const double tol = 128.0 * 2.220446049250313080847e-16 * scale * scale * scale;
    if (!(scale > 0.0) || !isfinite(det) || fabs(det) <= tol) return 0;
    const double id = 1.0 / det;
    const S3 inv = {(m->yy * m->zz - m->yz * m->yz) * id,
                    (m->xx * m->zz - m->xz * m->xz) * id,
                    (m->xx * m->yy - m->xy * m->xy) * id,
                    (m->xz * m->yz - m->xy * m->zz) * id,
                    (m->xy * m->yz - m->xz * m->yy) * id,
                    (m->xy * m->xz - m->xx * m->yz) * id};
    *out = v3(inv.xx * rhs.x + inv.xy * rhs.y + inv.xz * rhs.z,
              inv.xy * rhs.x + inv.yy * rhs.y + inv.yz * rhs.z,
              inv.xz * rhs.x + inv.yz * rhs.y + inv.zz * rhs.z);
    return 1;
}
static int restore_momentum(swo_structure* s, const Momentum* target) {
    if (!(target->mass > 0.0)) return 1;
    Momentum cur = measure_momentum(s);
    const V3 dv = vdiv(sub(target->p, cur.p), target->mass);
    for (uint64_t i = 0; i < s->n; ++i)
        if (s->nodes[i].w > 0.0) s->nodes[i].v = add(s->nodes[i].v, dv);
    cur = measure_momentum(s);
    S3 I; memset(&I, 0, sizeof I);
    for (uint64_t i = 0; i < s->n; ++i) {
        const Node* n = &s->nodes[i];
        if (n->w <= 0.0) continue;
        const double m = 1.0 / n->w;
        const V3 r = sub(n->x, cur.com);
        I.xx += m * (r.y * r.y + r.z * r.z);
        I.yy += m * (r.x * r.x + r.z * r.z);
        I.zz += m * (r.x * r.x + r.y * r.y);
        I.xy -= m * r.x * r.y;
        I.xz -= m * r.x * r.z;
        I.yz -= m * r.y * r.z;
    }
    if (!spd(&I)) return 1;
    V3 w;
    if (!checked_solve(&I, sub(target->L, cur.L), &w))
        return 0; /* equilibrated fallback solve is not restated */
    for (uint64_t i = 0; i < s->n; ++i)
        if (s->nodes[i].w > 0.0)
            s->nodes[i].v = add(s->nodes[i].v, cross(w, sub(s->nodes[i].x, cur.com)));
    return 1;
}

/* ---------------- suspension (suspension.cpp) ---------------------------- */
static int endpoint_state(swo_structure* s, int node, int point, const M3* invI,
                          V3* pos, double* w, V3* offset, int* rigid, int* fixed) {
    *offset = v3(0, 0, 0);
    *rigid = 0;
    if (node >= 0) {
        *pos = s->nodes[node].x;
        *w = s->nodes[node].w;
        *fixed = s->nodes[node].w == 0.0;
        return 1;
    }
    (void)invI;
    if (!point_position(&s->pdef, &s->payload, s->hang_local[point], pos)) return 0;
    *offset = sub(*pos, s->payload.com);
    *rigid = 1;
    *fixed = 0; /* ground mode Free */
    *w = 1.0 / s->pdef.mass;
    return 1;
}

static double effective_inverse_mass(double w, int rigid, V3 offset, const M3* invI,
                                     V3 g) {
    double r = w;
    if (rigid && w > 0.0) {
        const V3 rot = cross(offset, g);
        r += dot(rot, m3v(invI, rot));
    }
    return r;
}

static swb_status line_iteration(swo_structure* s, double dt) {
    M3 I, invI;
    if (!world_inertia(&s->pdef, &s->payload, &I) || !m3inv(&I, &invI))
        return fail(SWB_SUSPENSION_ERROR, "payload inertia");
    for (uint64_t k = 0; k < s->nseg; ++k) {
        Segment* g = &s->seg[k];
        V3 fp, tp, fo, to;
        double fw, tw;
        int fr, ff, tr, tf;
        if (!endpoint_state(s, g->from_node, g->from_point, &invI, &fp, &fw, &fo, &fr, &ff) ||
            !endpoint_state(s, g->to_node, g->to_point, &invI, &tp, &tw, &to, &tr, &tf))
            return fail(SWB_SUSPENSION_ERROR, "line endpoint");
        const V3 diff = sub(tp, fp);
        const double l = len(diff);
        if (!isfinite(l) || l <= s->minimum_line_length)
            return fail(SWB_SUSPENSION_ERROR,
                        "line geometry is non-finite or scale-degenerate");
        const V3 dir = vdiv(diff, l);
        const V3 fg = dir;
        const V3 tg = neg(dir);
        /* projectUnilateralLine (suspension.cpp:1125-1163) */
        if (!(l > 0.0) || !(g->commanded > 0.0) || !(g->stiffness > 0.0) ||
            !(dt > 0.0) || !(g->lambda >= 0.0) || !isfinite(g->lambda) ||
            fabs(len(fg) - 1.0) > kUnitTolerance)
            return fail(SWB_SUSPENSION_ERROR, "invalid unilateral line projection input");
        const double eff = effective_inverse_mass(fw, fr && !ff, fo, &invI, fg) +
                           effective_inverse_mass(tw, tr && !tf, to, &invI, neg(fg));
        const double at = 1.0 / (g->stiffness * dt * dt);
        if (!(eff + at > 0.0))
            return fail(SWB_SUSPENSION_ERROR, "zero generalized effective mass");
        const double gap = g->commanded - l;
        const double cand = g->lambda + (-gap - at * g->lambda) / (eff + at);
        const double acc = 0.0 < cand ? cand : 0.0; /* std::max(0.0, cand) */
        const double inc = acc - g->lambda;
        g->lambda = acc;
        /* applyCorrection for both endpoints */
        for (int e = 0; e < 2; ++e) {
            const int node = e == 0 ? g->from_node : g->to_node;
            const double w = e == 0 ? fw : tw;
            const int fixed = e == 0 ? ff : tf;
            const V3 grad = e == 0 ? fg : tg;
            const V3 off = e == 0 ? fo : to;
            if (fixed) continue;
            if (node >= 0) {
                s->nodes[node].x = add(s->nodes[node].x, mul(grad, w * inc));
            } else {
                s->payload.com = add(s->payload.com, mul(grad, w * inc));
                const V3 rot = mul(m3v(&invI, cross(off, grad)), inc);
                Q qi;
                if (!qincrement(rot, &qi) ||
                    !qcanon(qmul(qi, s->payload.orientation), &s->payload.orientation))
                    return fail(SWB_SUSPENSION_ERROR, "rotation increment");
            }
        }
    }
    return SWB_OK;
}

static int endpoint_position(swo_structure* s, int node, int point, V3* out) {
    if (node >= 0) { *out = s->nodes[node].x; return 1; }
    return point_position(&s->pdef, &s->payload, s->hang_local[point], out);
}
static int endpoint_velocity(swo_structure* s, int node, int point, V3* out) {
    if (node >= 0) { *out = s->nodes[node].v; return 1; }
    return point_velocity(&s->pdef, &s->payload, s->hang_local[point], out);
}

static swb_status suspension_finish(swo_structure* s, double dt) {
    /* reconstructPayloadVelocity (suspension.cpp:2386-2411) */
    s->payload.linear_velocity = vdiv(sub(s->payload.com, s->previous_payload.com), dt);
    Q conj = {s->previous_payload.orientation.w, -s->previous_payload.orientation.x,
              -s->previous_payload.orientation.y, -s->previous_payload.orientation.z};
    Q delta;
    if (!qcanon(qmul(s->payload.orientation, conj), &delta))
        return fail(SWB_SUSPENSION_ERROR, "payload orientation");
    const double cw = delta.w < -1.0 ? -1.0 : (1.0 < delta.w ? 1.0 : delta.w);
    const double half = acos(cw);
    const double sn = sin(half);
    if (fabs(sn) < 1.0e-12) {
        s->payload.angular_velocity = mul(v3(delta.x, delta.y, delta.z), 2.0 / dt);
    } else {
        const V3 axis = v3(delta.x / sn, delta.y / sn, delta.z / sn);
        s->payload.angular_velocity = mul(axis, 2.0 * half / dt);
    }
    /* applyLineDamping (suspension.cpp:2413-2479) */
    M3 I, invI;
    if (!world_inertia(&s->pdef, &s->payload, &I) || !m3inv(&I, &invI))
        return fail(SWB_SUSPENSION_ERROR, "payload inertia");
    for (uint64_t k = 0; k < s->nseg; ++k) {
        Segment* g = &s->seg[k];
        if (!(g->lambda > 0.0) || !(g->damping > 0.0)) continue;
        V3 from, to, vf, vt;
        if (!endpoint_position(s, g->from_node, g->from_point, &from) ||
            !endpoint_position(s, g->to_node, g->to_point, &to))
            return fail(SWB_SUSPENSION_ERROR, "endpoint");
        const V3 dir = normalized(sub(to, from));
        if (!endpoint_velocity(s, g->to_node, g->to_point, &vt) ||
            !endpoint_velocity(s, g->from_node, g->from_point, &vf))
            return fail(SWB_SUSPENSION_ERROR, "endpoint");
        const double rel = dot(sub(vt, vf), dir);
        double eff = 0.0;
        if (g->from_node >= 0) eff += s->nodes[g->from_node].w;
        else {
            const V3 rxn = cross(sub(from, s->payload.com), dir);
            eff += 1.0 / s->pdef.mass + dot(rxn, m3v(&invI, rxn));
        }
        if (g->to_node >= 0) eff += s->nodes[g->to_node].w;
        else {
            const V3 rxn = cross(sub(to, s->payload.com), dir);
            eff += 1.0 / s->pdef.mass + dot(rxn, m3v(&invI, rxn));
        }
        if (!(eff > 0.0) || rel == 0.0) continue;
        /* boundedAxialDampingImpulse (suspension.cpp:1165-1185) */
        double mag = 0.0;
        if (!(g->damping == 0.0 || eff == 0.0 || rel == 0.0)) {
            const double req = g->damping * fabs(rel) * dt;
            const double stop = fabs(rel) / eff;
            mag = copysign(stop < req ? stop : req, rel);
        }
        const V3 fi = mul(dir, mag);
        const V3 ti = neg(fi);
        for (int e = 0; e < 2; ++e) {
            const int node = e == 0 ? g->from_node : g->to_node;
            const V3 point = e == 0 ? from : to;
            const V3 imp = e == 0 ? fi : ti;
            if (node >= 0) {
                if (s->nodes[node].w > 0.0)
                    s->nodes[node].v = add(s->nodes[node].v, mul(imp, s->nodes[node].w));
            } else {
                s->payload.linear_velocity =
                    add(s->payload.linear_velocity, vdiv(imp, s->pdef.mass));
                s->payload.angular_velocity = add(
                    s->payload.angular_velocity,
                    m3v(&invI, cross(sub(point, s->payload.com), imp)));
            }
        }
    }
    /* certifySubstep (suspension.cpp:2324-2359) */
    if (!finite3(s->payload.com) || !finiteq(s->payload.orientation) ||
        !finite3(s->payload.linear_velocity) || !finite3(s->payload.angular_velocity) ||
        fabs(qnorm2(s->payload.orientation) - 1.0) > 1.0e-12)
        return fail(SWB_SUSPENSION_ERROR, "payload trial state is non-finite or unnormalized");
    double maxres = 0.0;
    for (uint64_t k = 0; k < s->nseg; ++k) {
        Segment* g = &s->seg[k];
        V3 from, to;
        endpoint_position(s, g->from_node, g->from_point, &from);
        endpoint_position(s, g->to_node, g->to_point, &to);
        const double l = len(sub(to, from));
        if (!isfinite(l)) return fail(SWB_SUSPENSION_ERROR, "line trial length is non-finite");
        const double d0 = l - g->commanded;
        const double stretch = 0.0 < d0 ? d0 : 0.0;
        const double cs = g->lambda / (g->stiffness * dt * dt);
        const double r = fabs(stretch - cs);
        maxres = maxres < r ? r : maxres;
    }
    s->max_residual = maxres;
    if (maxres > s->maximum_line_residual) {
        snprintf(g_error, sizeof g_error,
                 "maximum line residual %.17g m exceeds configured bound %.17g m",
                 maxres, s->maximum_line_residual);
        return SWB_SUSPENSION_ERROR;
    }
    /* finishSubstep: payload line wrench (suspension.cpp:2582-2589) */
    s->line_force = v3(0, 0, 0);
    s->line_moment = v3(0, 0, 0);
    for (uint64_t k = 0; k < s->nseg; ++k) {
        Segment* g = &s->seg[k];
        V3 from, to;
        endpoint_position(s, g->from_node, g->from_point, &from);
        endpoint_position(s, g->to_node, g->to_point, &to);
        const V3 dir = normalized(sub(to, from));
        const V3 fimp = mul(dir, g->lambda / dt);
        const V3 timp = neg(fimp);
        if (g->from_point >= 0 || g->to_point >= 0) {
            const V3 imp = g->to_point >= 0 ? timp : fimp;
            const V3 pt = g->to_point >= 0 ? to : from;
            s->line_force = add(s->line_force, vdiv(imp, dt));
            s->line_moment = add(s->line_moment,
                                 cross(sub(pt, s->payload.com), vdiv(imp, dt)));
        }
    }
    return SWB_OK;
}

/* ---------------- step --------------------------------------------------- */
typedef struct {
    Node* nodes;
    Distance* dist;
    Dihedral* dih;
    Segment* seg;
    Membrane* mem;
    Payload payload, previous_payload;
} Saved;

/* The ground plane after each iteration: a free node below it goes back
 * onto it along the normal; with friction its motion along the plane since
 * the substep's start is stopped while it is at most friction x the
 * correction, else shortened by that length. */
static void ground_pass(swo_structure* s) {
    const V3 n = s->ground_normal;
    for (uint64_t i = 0; i < s->n; ++i) {
        Node* p = &s->nodes[i];
        if (!(p->w > 0.0)) continue;
        const double c = dot(n, p->x) - s->ground_offset;
        if (!(c < 0.0)) continue;
        p->x = sub(p->x, smul(c, n));
        if (s->ground_friction > 0.0) {
            V3 d = sub(p->x, p->prev);
            d = sub(d, smul(dot(n, d), n));
            const double length = sqrt(dot(d, d)), limit = -s->ground_friction * c;
            const double k = length <= limit ? 1.0 : limit / length;
            p->x = sub(p->x, smul(k, d));
        }
    }
}

static int cmp_seg(const void* a, const void* b) {
    const uint64_t* x = (const uint64_t*)a;
    const uint64_t* y = (const uint64_t*)b;
    if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
    if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
    return 0;
}

swb_status swo_set_line_contact(swo_structure* s, const swb_line_contact* lc) {
    if (!lc || !lc->enabled) {
        s->lines = 0;
        return SWB_OK;
    }
    if (!s->line_seg) {
        uint64_t k = 0;
        s->line_seg = malloc((s->m + 1) * sizeof *s->line_seg);
        for (uint64_t i = 0; i < s->m; ++i)
            if (s->dist[i].kind == SWB_CONSTRAINT_CABLE) {
                const uint64_t a = s->dist[i].a, b = s->dist[i].b;
                s->line_seg[k][0] = a < b ? a : b;
                s->line_seg[k][1] = a < b ? b : a;
                ++k;
            }
        qsort(s->line_seg, k, sizeof *s->line_seg, cmp_seg);
        uint64_t u = 0;
        for (uint64_t i = 0; i < k; ++i)
            if (u == 0 || cmp_seg(s->line_seg[u - 1], s->line_seg[i]) != 0) {
                s->line_seg[u][0] = s->line_seg[i][0];
                s->line_seg[u][1] = s->line_seg[i][1];
                ++u;
            }
        s->nseg_lines = u;
    }
    s->lines = 1;
    s->line_radius = lc->radius;
    s->line_reach = lc->radius + 0.5 * lc->margin;
    return SWB_OK;
}

/* The substep's candidate pairs at the predicted positions: segments that
 * share no node and whose boxes, widened by the reach, overlap, in key
 * order. */
static void line_broadphase(swo_structure* s) {
    s->npairs = 0;
    const double r = s->line_reach;
    for (uint64_t i = 0; i < s->nseg_lines; ++i) {
        const V3 a = s->nodes[s->line_seg[i][0]].x, b = s->nodes[s->line_seg[i][1]].x;
        for (uint64_t j = i + 1; j < s->nseg_lines; ++j) {
            const uint64_t* q = s->line_seg[j];
            if (q[0] == s->line_seg[i][0] || q[0] == s->line_seg[i][1] || q[1] == s->line_seg[i][0] ||
                q[1] == s->line_seg[i][1])
                continue;
            const V3 c = s->nodes[q[0]].x, d = s->nodes[q[1]].x;
            if (fmin(a.x, b.x) - r > fmax(c.x, d.x) + r || fmin(c.x, d.x) - r > fmax(a.x, b.x) + r ||
                fmin(a.y, b.y) - r > fmax(c.y, d.y) + r || fmin(c.y, d.y) - r > fmax(a.y, b.y) + r ||
                fmin(a.z, b.z) - r > fmax(c.z, d.z) + r || fmin(c.z, d.z) - r > fmax(a.z, b.z) + r)
                continue;
            if (s->npairs == s->pairs_cap) {
                s->pairs_cap = s->pairs_cap ? 2 * s->pairs_cap : 64;
                s->line_pair = realloc(s->line_pair, s->pairs_cap * sizeof *s->line_pair);
            }
            s->line_pair[s->npairs][0] = i;
            s->line_pair[s->npairs][1] = j;
            ++s->npairs;
        }
    }
}

/* The candidates' projections in key order: the segments' closest points
 * (Ericson's segment-segment method) pushed apart to 2 x radius. */
static void line_project(swo_structure* s) {
    const double gap = 2.0 * s->line_radius;
    for (uint64_t k = 0; k < s->npairs; ++k) {
        Node* A = &s->nodes[s->line_seg[s->line_pair[k][0]][0]];
        Node* B = &s->nodes[s->line_seg[s->line_pair[k][0]][1]];
        Node* C = &s->nodes[s->line_seg[s->line_pair[k][1]][0]];
        Node* D = &s->nodes[s->line_seg[s->line_pair[k][1]][1]];
        const V3 d1 = sub(B->x, A->x), d2 = sub(D->x, C->x), r = sub(A->x, C->x);
        const double eps = 1.0e-12;
        const double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
        double ps = 0.0, pt = 0.0;
        if (a <= eps && e <= eps) {
        } else if (a <= eps) {
            pt = fmin(fmax(f / e, 0.0), 1.0);
        } else {
            const double c = dot(d1, r);
            if (e <= eps) {
                ps = fmin(fmax(-c / a, 0.0), 1.0);
            } else {
                const double b = dot(d1, d2), denom = a * e - b * b;
                ps = denom != 0.0 ? fmin(fmax((b * f - c * e) / denom, 0.0), 1.0) : 0.0;
                pt = (b * ps + f) / e;
                if (pt < 0.0) {
                    pt = 0.0;
                    ps = fmin(fmax(-c / a, 0.0), 1.0);
                } else if (pt > 1.0) {
                    pt = 1.0;
                    ps = fmin(fmax((b - c) / a, 0.0), 1.0);
                }
            }
        }
        const V3 diff = sub(add(A->x, smul(ps, d1)), add(C->x, smul(pt, d2)));
        const double dist = sqrt(dot(diff, diff));
        if (!(dist < gap) || !(dist > 0.0)) continue;
        const V3 n = smul(1.0 / dist, diff);
        const double wa = A->w * (1.0 - ps), wb = B->w * ps, wc = C->w * (1.0 - pt), wd = D->w * pt;
        const double W = wa * (1.0 - ps) + wb * ps + wc * (1.0 - pt) + wd * pt;
        if (!(W > 0.0)) continue;
        const double dl = (gap - dist) / W;
        A->x = add(A->x, smul(wa * dl, n));
        B->x = add(B->x, smul(wb * dl, n));
        C->x = sub(C->x, smul(wc * dl, n));
        D->x = sub(D->x, smul(wd * dl, n));
    }
}

swb_status swo_set_ground(swo_structure* s, const swb_ground* g) {
    if (!g || !g->enabled) {
        s->ground = 0;
        return SWB_OK;
    }
    s->ground = 1;
    s->ground_normal = fromabi(g->normal);
    s->ground_offset = g->offset;
    s->ground_friction = g->friction;
    return SWB_OK;
}

static swb_status substep(swo_structure* s, double dt, const swb_step_settings* st) {
    const V3 g = fromabi(st->gravity);
    pressure_scatter(s);
    if (s->has_suspension) {
        s->previous_payload = s->payload;
        for (uint64_t k = 0; k < s->nseg; ++k) {
            s->seg[k].lambda = 0.0;
            s->seg[k].commanded = s->seg[k].rest;
        }
        /* appliedWrench is zero through the adapter */
        const V3 total = add(v3(0, 0, 0), smul(s->pdef.mass, g));
        if (!integrate_payload(&s->pdef, &s->payload, dt, total, v3(0, 0, 0)))
            return fail(SWB_SUSPENSION_ERROR, "payload integration");
    }
    const double damping = exp(-st->velocity_damping * dt);
    predict(s, dt, g, damping, fromabi(st->damping_reference_velocity));
    if (s->lines) line_broadphase(s);
    int preserve = !s->has_suspension && (s->h > 0 || s->nm > 0);
    for (uint64_t i = 0; preserve && i < s->n; ++i)
        if (!(s->nodes[i].w > 0.0)) preserve = 0;
    Momentum predicted; memset(&predicted, 0, sizeof predicted);
    if (preserve) predicted = measure_momentum(s);
    for (uint64_t i = 0; i < s->m; ++i) s->dist[i].lambda = 0.0;
    for (uint64_t i = 0; i < s->nm; ++i) {
        s->mem[i].multiplier = v3(0, 0, 0);
        s->mem[i].residual = 0.0;
    }
    for (uint64_t i = 0; i < s->h; ++i) s->dih[i].lambda = 0.0;
    const double inv_dt2 = 1.0 / (dt * dt);
    /* three quarters of the cable pairs close the substep, the rest run
     * before the general sweeps of the first iterations (soft_body.cpp:1288-1317) */
    const int pairs = st->cable_sweep_pairs;
    const int closing = pairs > 0 ? pairs - pairs / 4 : 0;
    const int interleaved = pairs - closing;
    const int iters = st->constraint_iterations > 1 ? st->constraint_iterations : 1;
    for (int it = 0; it < st->constraint_iterations; ++it) {
        const int cable_pairs = interleaved / iters + (it < interleaved % iters ? 1 : 0);
        for (int q = 0; q < cable_pairs; ++q) cable_pair(s, inv_dt2);
        for (uint64_t i = 0; i < s->m; ++i) project_distance(s, &s->dist[i], inv_dt2);
        for (uint64_t i = 0; i < s->nm; ++i)
            if (!solve_membrane(s, &s->mem[i], dt))
                return fail(SWB_INVALID_ARGUMENT, "membrane system is singular or its right-hand side not finite");
        for (uint64_t i = 0; i < s->h; ++i) solve_dihedral(s, &s->dih[i], inv_dt2);
        if (s->has_suspension) {
            swb_status r = line_iteration(s, dt);
            if (r != SWB_OK) return r;
        }
        if (s->lines) line_project(s);
        if (s->ground) ground_pass(s);
    }
    if (st->constraint_iterations > 0)
        for (int q = 0; q < closing; ++q) cable_pair(s, inv_dt2);
    else
        for (int q = 0; q < pairs; ++q) cable_pair(s, inv_dt2);
    if (st->constraint_iterations > 0)
        for (uint64_t i = 0; i < s->m; ++i)
            if (s->dist[i].kind == SWB_CONSTRAINT_SEAM_STITCH)
                project_distance(s, &s->dist[i], inv_dt2);
    for (uint64_t i = 0; i < s->nm; ++i) membrane_residual(s, &s->mem[i], dt);
    finalize(s, dt);
    if (preserve && !restore_momentum(s, &predicted))
        return fail(SWB_UNSUPPORTED, "ill-conditioned momentum solve not restated");
    if (s->has_suspension) return suspension_finish(s, dt);
    return SWB_OK;
}

swb_status swo_step(swo_structure* s, const swb_step_settings* st) {
    if (!(st->time_step > 0.0) || !isfinite(st->time_step) || st->substeps <= 0 ||
        st->constraint_iterations < 0 || st->cable_sweep_pairs < 0 ||
        st->velocity_damping < 0.0 || !isfinite(st->velocity_damping) ||
        !finite3(fromabi(st->gravity)) || !finite3(fromabi(st->damping_reference_velocity)))
        return fail(SWB_INVALID_ARGUMENT, "Invalid SoftBody step settings");
    if (s->has_suspension) {
        if (st->constraint_iterations == 0)
            return fail(SWB_INVALID_ARGUMENT, "Invalid coupled SoftBody step settings");
        if (st->constraint_iterations != s->line_iterations)
            return fail(SWB_INVALID_ARGUMENT,
                        "Coupled structural iterations must equal the registered "
                        "suspension lineIterations contract");
    }
    /* transactional: snapshot the whole state (structure.cpp:807-831) */
    Saved sv;
    sv.nodes = malloc((s->n ? s->n : 1) * sizeof(Node));
    memcpy(sv.nodes, s->nodes, s->n * sizeof(Node));
    sv.seg = malloc((s->nseg ? s->nseg : 1) * sizeof(Segment));
    if (s->nseg) memcpy(sv.seg, s->seg, s->nseg * sizeof(Segment));
    sv.mem = malloc((s->nm ? s->nm : 1) * sizeof(Membrane));
    if (s->nm) memcpy(sv.mem, s->mem, s->nm * sizeof(Membrane));
    sv.payload = s->payload;
    sv.previous_payload = s->previous_payload;
    const double dt = st->time_step / st->substeps;
    swb_status status = SWB_OK;
    for (int k = 0; k < st->substeps && status == SWB_OK; ++k) {
        for (uint64_t i = 0; i < s->n; ++i) s->nodes[i].force = s->pending[i];
        status = substep(s, dt, st);
    }
    if (status != SWB_OK) {
        memcpy(s->nodes, sv.nodes, s->n * sizeof(Node));
        if (s->nseg) memcpy(s->seg, sv.seg, s->nseg * sizeof(Segment));
        if (s->nm) memcpy(s->mem, sv.mem, s->nm * sizeof(Membrane));
        s->payload = sv.payload;
        s->previous_payload = sv.previous_payload;
    } else {
        V3 applied = v3(0, 0, 0);
        for (uint64_t i = 0; i < s->n; ++i) {
            applied = add(applied, s->pending[i]);
            s->pending[i] = v3(0, 0, 0);
            s->nodes[i].force = v3(0, 0, 0);
        }
        s->last_applied = applied;
        s->accepted += 1;
        s->time += st->time_step;
    }
    free(sv.nodes);
    free(sv.seg);
    free(sv.mem);
    return status;
}

/* Structure::diagnostics (structure.cpp:833-959), without membranes and
 * contact. */
swb_status swo_diagnostics(const swo_structure* s, swb_diagnostics* o) {
    memset(o, 0, sizeof *o);
    o->node_count = s->n;
    o->triangle_count = s->t;
    o->constraint_count = s->m;
    o->dihedral_count = s->h;
    int fin = 1;
    V3 wp = v3(0, 0, 0), p = v3(0, 0, 0);
    double mass = 0.0, ke = 0.0;
    for (uint64_t i = 0; i < s->n; ++i) {
        const Node* n = &s->nodes[i];
        fin = fin && finite3(n->x) && finite3(n->prev) && finite3(n->v) &&
              isfinite(n->w) && n->w >= 0.0;
        if (n->w > 0.0) {
            const double m = 1.0 / n->w;
            o->dynamic_node_count += 1;
            mass += m;
            wp = add(wp, mul(n->x, m));
            p = add(p, mul(n->v, m));
            ke += 0.5 * m * dot(n->v, n->v);
        }
    }
    V3 com = v3(0, 0, 0);
    if (mass > 0.0) com = mul(wp, 1.0 / mass);
    if (s->has_suspension) {
        const double m = s->pdef.mass;
        const V3 mom = smul(m, s->payload.linear_velocity);
        wp = add(wp, mul(s->payload.com, m));
        mass += m;
        com = mul(wp, 1.0 / mass);
        p = add(p, mom);
        M3 I;
        world_inertia(&s->pdef, &s->payload, &I);
        const V3 L = m3v(&I, s->payload.angular_velocity);
        ke += 0.5 * m * dot(s->payload.linear_velocity, s->payload.linear_velocity) +
              0.5 * dot(s->payload.angular_velocity, L);
        o->suspension_segment_count = s->nseg;
        o->maximum_suspension_residual = s->max_residual;
        fin = fin && finite3(s->payload.com) && finite3(mom);
    }
    o->total_dynamic_mass = mass;
    o->center_of_mass = toabi(com);
    o->linear_momentum = toabi(p);
    o->kinetic_energy = ke;
    double maxd = 0.0, maxc = 0.0;
    for (uint64_t i = 0; i < s->m; ++i) {
        const Distance* c = &s->dist[i];
        const double l = len(sub(s->nodes[c->b].x, s->nodes[c->a].x));
        const double e = l - c->rest;
        if (c->kind == SWB_CONSTRAINT_CABLE) {
            const double ex = 0.0 < e ? e : 0.0;
            maxc = maxc < ex ? ex : maxc;
        } else {
            maxd = maxd < fabs(e) ? fabs(e) : maxd;
        }
    }
    o->maximum_distance_error = maxd;
    o->maximum_cable_extension = maxc;
    /* membrane strain at the current positions and the last substep's
     * residual (structure.cpp:924-939, membrane diagnostics soft_body.cpp:204-270) */
    o->membrane_count = s->nm;
    double max_strain = 0.0, max_residual = 0.0;
    for (uint64_t i = 0; i < s->nm; ++i) {
        const Membrane* e = &s->mem[i];
        V3 g[3][3];
        const V3 strain = membrane_strain(s->nodes, e, g);
        const S3 k = effective_stiffness(e, strain);
        const V3 resultant = s3v(&k, strain);
        const double energy = 0.5 * e->area * dot(strain, resultant);
        double a = fabs(strain.x);
        a = fabs(strain.y) > a ? fabs(strain.y) : a;
        a = fabs(strain.z) > a ? fabs(strain.z) : a;
        max_strain = a > max_strain ? a : max_strain;
        max_residual = fabs(e->residual) > max_residual ? fabs(e->residual) : max_residual;
        fin = fin && isfinite(energy) && isfinite(e->residual);
    }
    o->maximum_absolute_membrane_strain = max_strain;
    o->maximum_membrane_residual = max_residual;
    V3 pend = v3(0, 0, 0);
    for (uint64_t i = 0; i < s->n; ++i) pend = add(pend, s->pending[i]);
    o->pending_external_force = toabi(pend);
    o->last_applied_external_force = toabi(s->last_applied);
    o->finite = fin && finite3(com) && finite3(p) && isfinite(ke) ? 1u : 0u;
    return SWB_OK;
}

swb_status swo_read_nodes(const swo_structure* s, swb_node_state* out, uint64_t n) {
    if (n != s->n) return fail(SWB_INVALID_ARGUMENT, "node count mismatch");
    for (uint64_t i = 0; i < n; ++i) {
        out[i].position = toabi(s->nodes[i].x);
        out[i].previous_position = toabi(s->nodes[i].prev);
        out[i].velocity = toabi(s->nodes[i].v);
    }
    return SWB_OK;
}

swb_status swo_write_nodes(swo_structure* s, const swb_node_state* in, uint64_t n) {
    if (n != s->n) return fail(SWB_INVALID_ARGUMENT, "node count mismatch");
    for (uint64_t i = 0; i < n; ++i) {
        s->nodes[i].x = fromabi(in[i].position);
        s->nodes[i].prev = fromabi(in[i].previous_position);
        s->nodes[i].v = fromabi(in[i].velocity);
    }
    return SWB_OK;
}

swb_status swo_read_payload(const swo_structure* s, swb_payload_state* p, swb_wrench* w,
                            double* max_residual) {
    if (!s->has_suspension) return fail(SWB_INVALID_ARGUMENT, "no suspension");
    p->center_of_mass = toabi(s->payload.com);
    p->body_to_world.w = s->payload.orientation.w;
    p->body_to_world.x = s->payload.orientation.x;
    p->body_to_world.y = s->payload.orientation.y;
    p->body_to_world.z = s->payload.orientation.z;
    p->linear_velocity = toabi(s->payload.linear_velocity);
    p->angular_velocity = toabi(s->payload.angular_velocity);
    if (w) { w->force = toabi(s->line_force); w->moment = toabi(s->line_moment); }
    if (max_residual) *max_residual = s->max_residual;
    return SWB_OK;
}

swb_status swo_write_payload(swo_structure* s, const swb_payload_state* p) {
    if (!s->has_suspension) return fail(SWB_INVALID_ARGUMENT, "no suspension");
    s->payload.com = fromabi(p->center_of_mass);
    s->payload.orientation.w = p->body_to_world.w;
    s->payload.orientation.x = p->body_to_world.x;
    s->payload.orientation.y = p->body_to_world.y;
    s->payload.orientation.z = p->body_to_world.z;
    s->payload.linear_velocity = fromabi(p->linear_velocity);
    s->payload.angular_velocity = fromabi(p->angular_velocity);
    return SWB_OK;
}

/* Segment tension in definition order (tension = lambda/dt^2 of the last
 * substep, suspension.cpp:2533). */
swb_status swo_read_segment_lambdas(const swo_structure* s, double* out, uint64_t n) {
    if (n != s->nseg) return fail(SWB_INVALID_ARGUMENT, "segment count mismatch");
    for (uint64_t k = 0; k < s->nseg; ++k) out[s->seg[k].definition_index] = s->seg[k].lambda;
    return SWB_OK;
}

/* The dihedral evaluation alone, for the analytic-gradient known-answer
 * tests (softwing_material_test.cpp:182-362). out: angle, 12 gradient
 * components, valid flag. */
void swo_evaluate_dihedral(const double* p12, double* out14) {
    const DihedralEval e = evaluate_dihedral(v3(p12[0], p12[1], p12[2]),
                                             v3(p12[3], p12[4], p12[5]),
                                             v3(p12[6], p12[7], p12[8]),
                                             v3(p12[9], p12[10], p12[11]));
    out14[0] = e.angle;
    for (int k = 0; k < 4; ++k) {
        out14[1 + 3 * k] = e.g[k].x;
        out14[2 + 3 * k] = e.g[k].y;
        out14[3 + 3 * k] = e.g[k].z;
    }
    out14[13] = e.valid ? 1.0 : 0.0;
}
