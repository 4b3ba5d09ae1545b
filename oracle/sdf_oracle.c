/*
 * sdf_oracle.c — FP64 CPU restatement of the reference triangle-mesh SDF
 * (src/fluid/SDFBoundary.cpp) and of the fluid-to-mesh contact-force
 * reduction (src/main.cpp:557-571,604-710).
 *
 * TEST INFRASTRUCTURE ONLY (see pbf_oracle.h).  The reference code is C++
 * over Eigen; Eigen/Core is missing from the reference's vendored tree, so it
 * cannot be compiled here and this file restates it in plain C.
 */
#include "pbf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { orc_real x, y, z; } d3;
static inline d3 mk(orc_real x, orc_real y, orc_real z) { d3 r = {x, y, z}; return r; }
static inline d3 sub(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 add(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 scl(d3 a, orc_real s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline orc_real dt3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 crs(d3 a, d3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline orc_real nrm(d3 a) { return sqrt(dt3(a, a)); }
static inline d3 dmin(d3 a, d3 b) { return mk(fmin(a.x, b.x), fmin(a.y, b.y), fmin(a.z, b.z)); }
static inline d3 dmax(d3 a, d3 b) { return mk(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)); }
static inline orc_real comp(d3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }

/* Feature enum (SDFBoundary.cpp:17) */
enum { F_FACE, F_EDGE_AB, F_EDGE_AC, F_EDGE_BC, F_VA, F_VB, F_VC };

/* closestPointOnTriangle, Ericson 5.1.5 with feature (SDFBoundary.cpp:22-54) */
static d3 closest_on_tri(d3 P, d3 A, d3 B, d3 C, int* feature)
{
    const d3 AB = sub(B, A), AC = sub(C, A), AP = sub(P, A);
    const orc_real d1 = dt3(AB, AP), d2 = dt3(AC, AP);
    if (d1 <= 0 && d2 <= 0) { *feature = F_VA; return A; }
    const d3 BP = sub(P, B);
    const orc_real d3_ = dt3(AB, BP), d4 = dt3(AC, BP);
    if (d3_ >= 0 && d4 <= d3_) { *feature = F_VB; return B; }
    const d3 CP = sub(P, C);
    const orc_real d5 = dt3(AB, CP), d6 = dt3(AC, CP);
    if (d6 >= 0 && d5 <= d6) { *feature = F_VC; return C; }
    const orc_real vc = d1 * d4 - d3_ * d2;
    if (vc <= 0 && d1 >= 0 && d3_ <= 0) { *feature = F_EDGE_AB; return add(A, scl(AB, d1 / (d1 - d3_))); }
    const orc_real vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) { *feature = F_EDGE_AC; return add(A, scl(AC, d2 / (d2 - d6))); }
    const orc_real va = d3_ * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3_) >= 0 && (d5 - d6) >= 0) {
        *feature = F_EDGE_BC;
        return add(B, scl(sub(C, B), (d4 - d3_) / ((d4 - d3_) + (d5 - d6))));
    }
    const orc_real denom = 1.0 / (va + vb + vc);
    *feature = F_FACE;
    return add(A, add(scl(AB, vb * denom), scl(AC, vc * denom)));
}

/* Tri with per-feature pseudo-normals (SDFBoundary.cpp:59-64) */
typedef struct {
    d3 A, B, C;
    int iA, iB, iC;
    d3 fn, eAB, eAC, eBC;
} tri_t;

typedef struct {
    d3 bmin, bmax;
    int start, count, left, right;
} node_t;

struct orc_mesh {
    int nv, nf;
    tri_t* tris;
    d3* vn; /* angle-weighted vertex normals */
    /* TriangleBVH (SDFBoundary.cpp:78-265) */
    node_t* nodes;
    int nnodes;
    int* order;
    d3 *tmin, *tmax, *cen;
    /* grid */
    orc_real origin[3], cell;
    int dims[3];
};

static void tri_set(tri_t* t, const orc_real* v)
{
    t->A = mk(v[3 * t->iA], v[3 * t->iA + 1], v[3 * t->iA + 2]);
    t->B = mk(v[3 * t->iB], v[3 * t->iB + 1], v[3 * t->iB + 2]);
    t->C = mk(v[3 * t->iC], v[3 * t->iC + 1], v[3 * t->iC + 2]);
    d3 n = crs(sub(t->B, t->A), sub(t->C, t->A));
    const orc_real len = nrm(n);
    if (len > 1e-12) n = scl(n, 1.0 / len);
    t->fn = n;
}

/* quickselect on order[lo, hi) by centroid axis (std::nth_element role in
 * SDFBoundary.cpp:212-216) */
static void nth_select(struct orc_mesh* m, int lo, int hi, int nth, int axis)
{
    int* o = m->order;
    while (hi - lo > 1) {
        const orc_real pv = comp(m->cen[o[lo + (hi - lo) / 2]], axis);
        int i = lo, j = hi - 1;
        while (i <= j) {
            while (comp(m->cen[o[i]], axis) < pv) ++i;
            while (comp(m->cen[o[j]], axis) > pv) --j;
            if (i <= j) { int t = o[i]; o[i] = o[j]; o[j] = t; ++i; --j; }
        }
        if (nth <= j) hi = j + 1;
        else if (nth >= i) lo = i;
        else return;
    }
}

/* buildRecursive (SDFBoundary.cpp:181-223) */
static int build_rec(struct orc_mesh* m, int start, int count)
{
    const int idx = m->nnodes++;
    d3 bmin = mk(1e30, 1e30, 1e30), bmax = mk(-1e30, -1e30, -1e30);
    d3 cmin = bmin, cmax = bmax;
    for (int i = start; i < start + count; ++i) {
        const int t = m->order[i];
        bmin = dmin(bmin, m->tmin[t]);
        bmax = dmax(bmax, m->tmax[t]);
        cmin = dmin(cmin, m->cen[t]);
        cmax = dmax(cmax, m->cen[t]);
    }
    m->nodes[idx].bmin = bmin;
    m->nodes[idx].bmax = bmax;
    m->nodes[idx].start = start;
    m->nodes[idx].count = count;
    m->nodes[idx].left = m->nodes[idx].right = -1;
    if (count <= 4) return idx; /* kLeafSize = 4 (:158) */
    const d3 ext = sub(cmax, cmin);
    int axis = 0;
    if (ext.y > ext.x) axis = 1;
    if (ext.z > comp(ext, axis)) axis = 2;
    const int mid = count / 2;
    nth_select(m, start, start + count, start + mid, axis);
    const int l = build_rec(m, start, mid);
    const int r = build_rec(m, start + mid, count - mid);
    m->nodes[idx].left = l;
    m->nodes[idx].right = r;
    return idx;
}

static void tri_aabbs(struct orc_mesh* m)
{
    for (int i = 0; i < m->nf; ++i) {
        const tri_t* t = &m->tris[i];
        m->tmin[i] = dmin(dmin(t->A, t->B), t->C);
        m->tmax[i] = dmax(dmax(t->A, t->B), t->C);
    }
}

typedef struct { int a, b, t; } edge_t;
static int edge_cmp(const void* x, const void* y)
{
    const edge_t* e = (const edge_t*)x;
    const edge_t* f = (const edge_t*)y;
    if (e->a != f->a) return e->a < f->a ? -1 : 1;
    if (e->b != f->b) return e->b < f->b ? -1 : 1;
    return e->t < f->t ? -1 : (e->t > f->t);
}

orc_mesh* orc_mesh_build(const orc_real* verts, int32_t nv, const int32_t* faces, int32_t nf, orc_real cell)
{
    struct orc_mesh* m = (struct orc_mesh*)calloc(1, sizeof(struct orc_mesh));
    m->nv = nv;
    m->nf = nf;
    /* grid AABB + 5-cell buffer (SDFBoundary.cpp:291-308) */
    d3 bmin = mk(1e30, 1e30, 1e30), bmax = mk(-1e30, -1e30, -1e30);
    for (int i = 0; i < nv; ++i) {
        const d3 v = mk(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
        bmin = dmin(bmin, v);
        bmax = dmax(bmax, v);
    }
    const orc_real buffer = cell * 5.0;
    m->origin[0] = bmin.x - buffer;
    m->origin[1] = bmin.y - buffer;
    m->origin[2] = bmin.z - buffer;
    m->cell = cell;
    const orc_real span[3] = {(bmax.x + buffer) - m->origin[0], (bmax.y + buffer) - m->origin[1],
                            (bmax.z + buffer) - m->origin[2]};
    for (int k = 0; k < 3; ++k) m->dims[k] = (int)ceil(span[k] / cell);

    /* triangles + face normals (:322-337) */
    m->tris = (tri_t*)calloc((size_t)nf, sizeof(tri_t));
    for (int f = 0; f < nf; ++f) {
        tri_t* t = &m->tris[f];
        t->iA = faces[3 * f];
        t->iB = faces[3 * f + 1];
        t->iC = faces[3 * f + 2];
        tri_set(t, verts);
        t->eAB = t->eAC = t->eBC = t->fn;
    }
    /* angle-weighted vertex normals (:341-358) */
    m->vn = (d3*)calloc((size_t)nv, sizeof(d3));
    for (int f = 0; f < nf; ++f) {
        const tri_t* t = &m->tris[f];
        const int iv[3] = {t->iA, t->iB, t->iC};
        const d3 P[3] = {t->A, t->B, t->C};
        for (int c = 0; c < 3; ++c) {
            const d3 vtx = P[c], p1 = P[(c + 1) % 3], p2 = P[(c + 2) % 3];
            d3 a = sub(p1, vtx), b = sub(p2, vtx);
            const orc_real la = nrm(a), lb = nrm(b);
            /* Eigen normalized() leaves a zero vector unchanged */
            if (la > 0) a = scl(a, 1.0 / la);
            if (lb > 0) b = scl(b, 1.0 / lb);
            orc_real cs = dt3(a, b);
            cs = cs < -1.0 ? -1.0 : (cs > 1.0 ? 1.0 : cs);
            const orc_real ang = acos(cs);
            m->vn[iv[c]] = add(m->vn[iv[c]], scl(t->fn, ang));
        }
    }
    for (int i = 0; i < nv; ++i) {
        const orc_real len = nrm(m->vn[i]);
        if (len > 1e-12) m->vn[i] = scl(m->vn[i], 1.0 / len);
    }
    /* edge pseudo-normals: average of exactly two incident faces (:361-383) */
    edge_t* e = (edge_t*)malloc(sizeof(edge_t) * 3 * (size_t)nf);
    for (int f = 0; f < nf; ++f) {
        const tri_t* t = &m->tris[f];
        const int pr[3][2] = {{t->iA, t->iB}, {t->iA, t->iC}, {t->iB, t->iC}};
        for (int c = 0; c < 3; ++c) {
            e[3 * f + c].a = pr[c][0] < pr[c][1] ? pr[c][0] : pr[c][1];
            e[3 * f + c].b = pr[c][0] < pr[c][1] ? pr[c][1] : pr[c][0];
            e[3 * f + c].t = f;
        }
    }
    qsort(e, 3 * (size_t)nf, sizeof(edge_t), edge_cmp);
    for (size_t i = 0; i < 3 * (size_t)nf;) {
        size_t j = i;
        while (j < 3 * (size_t)nf && e[j].a == e[i].a && e[j].b == e[i].b) ++j;
        if (j - i == 2) {
            const d3 s = add(m->tris[e[i].t].fn, m->tris[e[i + 1].t].fn);
            const orc_real len = nrm(s);
            if (len >= 1e-12) {
                const d3 en = scl(s, 1.0 / len);
                for (size_t k = i; k < j; ++k) {
                    tri_t* t = &m->tris[e[k].t];
                    const int a = e[k].a, b = e[k].b;
                    const int mnAB = t->iA < t->iB ? t->iA : t->iB, mxAB = t->iA < t->iB ? t->iB : t->iA;
                    const int mnAC = t->iA < t->iC ? t->iA : t->iC, mxAC = t->iA < t->iC ? t->iC : t->iA;
                    if (mnAB == a && mxAB == b) t->eAB = en;
                    else if (mnAC == a && mxAC == b) t->eAC = en;
                    else t->eBC = en;
                }
            }
        }
        i = j;
    }
    free(e);
    /* BVH (TriangleBVH::build, :87-106) */
    m->order = (int*)malloc(sizeof(int) * (size_t)(nf > 0 ? nf : 1));
    m->tmin = (d3*)malloc(sizeof(d3) * (size_t)(nf > 0 ? nf : 1));
    m->tmax = (d3*)malloc(sizeof(d3) * (size_t)(nf > 0 ? nf : 1));
    m->cen = (d3*)malloc(sizeof(d3) * (size_t)(nf > 0 ? nf : 1));
    for (int i = 0; i < nf; ++i) {
        m->order[i] = i;
        const tri_t* t = &m->tris[i];
        m->cen[i] = scl(add(add(t->A, t->B), t->C), 1.0 / 3.0);
    }
    tri_aabbs(m);
    m->nodes = (node_t*)malloc(sizeof(node_t) * 2 * (size_t)(nf > 0 ? nf : 1));
    m->nnodes = 0;
    if (nf > 0) build_rec(m, 0, nf);
    return m;
}

void orc_mesh_free(orc_mesh* m)
{
    if (!m) return;
    free(m->tris); free(m->vn); free(m->nodes); free(m->order); free(m->tmin); free(m->tmax); free(m->cen);
    free(m);
}

/* updateGeometryAndRefit + TriangleBVH::refit (SDFBoundary.cpp:120-148,438-453) */
void orc_mesh_refit(orc_mesh* m, const orc_real* verts)
{
    for (int f = 0; f < m->nf; ++f) tri_set(&m->tris[f], verts);
    tri_aabbs(m);
    for (int i = m->nnodes - 1; i >= 0; --i) {
        node_t* nd = &m->nodes[i];
        if (nd->left == -1) {
            d3 bmin = mk(1e30, 1e30, 1e30), bmax = mk(-1e30, -1e30, -1e30);
            for (int k = nd->start; k < nd->start + nd->count; ++k) {
                bmin = dmin(bmin, m->tmin[m->order[k]]);
                bmax = dmax(bmax, m->tmax[m->order[k]]);
            }
            nd->bmin = bmin;
            nd->bmax = bmax;
        } else {
            nd->bmin = dmin(m->nodes[nd->left].bmin, m->nodes[nd->right].bmin);
            nd->bmax = dmax(m->nodes[nd->left].bmax, m->nodes[nd->right].bmax);
        }
    }
}

void orc_mesh_grid_info(const orc_mesh* m, int32_t dims[3], orc_real origin[3], orc_real* cell)
{
    for (int k = 0; k < 3; ++k) { dims[k] = m->dims[k]; origin[k] = m->origin[k]; }
    *cell = m->cell;
}

typedef struct { orc_real dist2; d3 point; int feature, tri; } hit_t;

static orc_real sq_dist_aabb(d3 p, d3 bmin, d3 bmax)
{
    orc_real d2 = 0.0;
    for (int i = 0; i < 3; ++i) {
        const orc_real v = comp(p, i), lo = comp(bmin, i), hi = comp(bmax, i);
        if (v < lo) { const orc_real t = lo - v; d2 += t * t; }
        else if (v > hi) { const orc_real t = v - hi; d2 += t * t; }
    }
    return d2;
}

/* TriangleBVH::query (SDFBoundary.cpp:225-257) */
static void query(const struct orc_mesh* m, int ni, d3 P, hit_t* best)
{
    const node_t* nd = &m->nodes[ni];
    if (sq_dist_aabb(P, nd->bmin, nd->bmax) >= best->dist2) return;
    if (nd->left == -1) {
        for (int i = nd->start; i < nd->start + nd->count; ++i) {
            const int t = m->order[i];
            const tri_t* tr = &m->tris[t];
            int feat;
            const d3 cp = closest_on_tri(P, tr->A, tr->B, tr->C, &feat);
            const d3 dd = sub(P, cp);
            const orc_real d2 = dt3(dd, dd);
            if (d2 < best->dist2) {
                best->dist2 = d2;
                best->point = cp;
                best->feature = feat;
                best->tri = t;
            }
        }
        return;
    }
    const orc_real dL = sq_dist_aabb(P, m->nodes[nd->left].bmin, m->nodes[nd->left].bmax);
    const orc_real dR = sq_dist_aabb(P, m->nodes[nd->right].bmin, m->nodes[nd->right].bmax);
    if (dL <= dR) {
        if (dL < best->dist2) query(m, nd->left, P, best);
        if (dR < best->dist2) query(m, nd->right, P, best);
    } else {
        if (dR < best->dist2) query(m, nd->right, P, best);
        if (dL < best->dist2) query(m, nd->left, P, best);
    }
}

static hit_t closest(const struct orc_mesh* m, d3 P)
{
    hit_t h;
    h.dist2 = 1e30;
    h.point = mk(0, 0, 0);
    h.feature = F_FACE;
    h.tri = -1;
    if (m->nnodes > 0) query(m, 0, P, &h);
    return h;
}

/* signedDistanceAt (SDFBoundary.cpp:400-419) */
orc_real orc_mesh_signed_distance(const orc_mesh* m, const orc_real p[3])
{
    const d3 P = mk(p[0], p[1], p[2]);
    const hit_t h = closest(m, P);
    if (h.tri < 0) return 0.0;
    const tri_t* t = &m->tris[h.tri];
    d3 pn;
    switch (h.feature) {
    case F_FACE: pn = t->fn; break;
    case F_EDGE_AB: pn = t->eAB; break;
    case F_EDGE_AC: pn = t->eAC; break;
    case F_EDGE_BC: pn = t->eBC; break;
    case F_VA: pn = m->vn[t->iA]; break;
    case F_VB: pn = m->vn[t->iB]; break;
    default: pn = m->vn[t->iC]; break;
    }
    const orc_real sign = (dt3(sub(P, h.point), pn) >= 0.0) ? 1.0 : -1.0;
    return sign * sqrt(h.dist2);
}

/* recomputeDistances (SDFBoundary.cpp:421-436) */
void orc_mesh_grid(const orc_mesh* m, float* out)
{
    const int dx = m->dims[0], dy = m->dims[1], dz = m->dims[2];
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 0; x < dx; ++x)
        for (int y = 0; y < dy; ++y)
            for (int z = 0; z < dz; ++z) {
                const orc_real P[3] = {m->origin[0] + x * m->cell, m->origin[1] + y * m->cell,
                                     m->origin[2] + z * m->cell};
                out[((int64_t)x * dy + y) * dz + z] = (float)orc_mesh_signed_distance(m, P);
            }
}

int32_t orc_mesh_closest(const orc_mesh* m, const orc_real p[3], orc_real point[3], orc_real* dist2)
{
    const hit_t h = closest(m, mk(p[0], p[1], p[2]));
    point[0] = h.point.x;
    point[1] = h.point.y;
    point[2] = h.point.z;
    *dist2 = h.dist2;
    return h.tri;
}

/* barycentric, clamped and renormalised (src/main.cpp:557-571) */
static void barycentric(d3 Pt, d3 A, d3 B, d3 C, orc_real* u, orc_real* v, orc_real* w)
{
    const d3 v0 = sub(B, A), v1 = sub(C, A), v2 = sub(Pt, A);
    const orc_real d00 = dt3(v0, v0), d01 = dt3(v0, v1), d11 = dt3(v1, v1);
    const orc_real d20 = dt3(v2, v0), d21 = dt3(v2, v1);
    const orc_real denom = d00 * d11 - d01 * d01;
    if (fabs(denom) < 1e-20) { *u = 1; *v = 0; *w = 0; return; }
    const orc_real vv = (d11 * d20 - d01 * d21) / denom;
    const orc_real ww = (d00 * d21 - d01 * d20) / denom;
    orc_real uu = 1.0 - vv - ww;
    uu = fmax(0.0, uu);
    orc_real vc = fmax(0.0, vv), wc = fmax(0.0, ww);
    const orc_real s = uu + vc + wc;
    if (s > 1e-20) { uu /= s; vc /= s; wc /= s; }
    *u = uu; *v = vc; *w = wc;
}

/* computeContactForces (src/main.cpp:604-710): per candidate the closest
 * triangle, skip beyond band, push direction, velocity-into-surface magnitude,
 * barycentric split.  Summed in candidate order. */
int32_t orc_contact_forces(const orc_mesh* m, const pbf_contact_candidate* cand, uint32_t count,
                           orc_real band, int use_vel, orc_real* forces)
{
    memset(forces, 0, sizeof(orc_real) * 3 * (size_t)m->nv);
    int32_t contacts = 0;
    for (uint32_t c = 0; c < count; ++c) {
        const d3 P = mk(cand[c].pos[0], cand[c].pos[1], cand[c].pos[2]);
        const d3 vel = mk(cand[c].vel[0], cand[c].vel[1], cand[c].vel[2]);
        const hit_t h = closest(m, P); /* :637 */
        if (h.tri < 0) continue;
        const d3 to = sub(h.point, P);
        const orc_real dist = nrm(to);
        if (dist > band) continue; /* :642 */
        const tri_t* t = &m->tris[h.tri];
        d3 dir;
        if (dist > 1e-6) dir = scl(to, 1.0 / dist); /* :651-657 */
        else {
            d3 n = crs(sub(t->B, t->A), sub(t->C, t->A));
            const orc_real l = nrm(n);
            if (l > 0) n = scl(n, 1.0 / l);
            dir = scl(n, -1.0);
        }
        orc_real mag = 1.0;
        if (use_vel) { /* :661-665 */
            mag = fmax(0.0, dt3(vel, dir));
            if (mag <= 0.0) continue;
        }
        orc_real u, v, w;
        barycentric(h.point, t->A, t->B, t->C, &u, &v, &w); /* :667-669 */
        const d3 F = scl(dir, mag);
        const int iv[3] = {t->iA, t->iB, t->iC};
        const orc_real wt[3] = {u, v, w};
        for (int k = 0; k < 3; ++k) { /* :671-673 */
            forces[3 * iv[k]] += F.x * wt[k];
            forces[3 * iv[k] + 1] += F.y * wt[k];
            forces[3 * iv[k] + 2] += F.z * wt[k];
        }
        ++contacts;
    }
    return contacts;
}
