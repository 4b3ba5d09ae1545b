/*
 * pbf_oracle.c — FP64 CPU restatement of the reference PBF substep.
 *
 * TEST INFRASTRUCTURE ONLY (see pbf_oracle.h).  Restates, in orc_real
 * precision, the math of the reference compute shaders under
 * resources/shaders/compute/ and of PBFluids::setParams/step
 * (src/fluid/PBFluids.cpp).  OpenMP-parallel over particles so that it also
 * serves as the timed CPU baseline.
 */
#include "pbf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static inline orc_real clampd(orc_real v, orc_real lo, orc_real hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline orc_real dot3(const orc_real* a, const orc_real* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* PBFluids::setParams + setBounds (src/fluid/PBFluids.cpp:39-109, 299-306). */
void orc_derive(const pbf_fluid_config* c, orc_real pad, orc_params* p)
{
    memset(p, 0, sizeof(*p));
    for (int a = 0; a < 3; ++a) {
        p->bmin[a] = (orc_real)c->bounds_min[a] + pad; /* PBFluids.cpp:303 */
        p->bmax[a] = (orc_real)c->bounds_max[a] - pad; /* PBFluids.cpp:304 */
        p->g[a] = c->gravity[a];
    }
    p->damping = clampd(c->bound_damping, 0.0, 1.0); /* PBFluids.cpp:305 */
    p->substeps = c->substep_iterations;
    p->dt = (orc_real)c->dt / (orc_real)c->substep_iterations; /* PBFluids.cpp:52 */
    const orc_real h = c->h;
    p->h = h;
    p->h2 = h * h;
    p->rho0 = c->rho0;
    p->eps = c->eps;
    /* wq = calcSCorrKernel((dq,0,0), h) = poly6 at dq (PBFluids.cpp:45-46,
     * Kernels.cpp:9-27,216-219) */
    {
        const orc_real dq = (orc_real)c->delta_q * h;
        const orc_real r2 = dq * dq;
        p->wq = (r2 > p->h2) ? 0.0 : (315.0 / (64.0 * M_PI)) / pow(h, 9.0) * pow(p->h2 - r2, 3.0);
    }
    p->k_corr = c->k_corr;
    p->n_corr = c->n_corr;
    p->viscosity = c->viscosity;
    p->cohesion = c->cohesion_strength;
    p->i_radius = c->interaction_radius;
    p->i_strength = c->interaction_strength;
    p->w0_self = (315.0 / (64.0 * M_PI)) / (h * h * h); /* PBFluids.cpp:83 */
    p->poly6 = 315.0 / (64.0 * M_PI * pow(h, 9.0));     /* PBFluids.cpp:86 */
    p->spiky = 45.0 / (M_PI * pow(h, 6.0));             /* PBFluids.cpp:89 */
    p->inv_rho0 = 1.0 / (orc_real)c->rho0;                /* PBFluids.cpp:92 */
    p->hash_size = c->hash_size;
    p->mask = c->hash_size - 1u; /* PBFluids.cpp:95 */
    p->scorr = c->enable_scorr ? 1u : 0u;
    p->visc_on = c->enable_viscosity ? 1u : 0u;
    p->vort_on = c->enable_vorticity ? 1u : 0u;
    p->vort_eps = c->vorticity_epsilon;
    p->apbf = c->enable_apbf ? 1u : 0u;
    p->min_lod = c->enable_apbf ? c->min_lod : c->solver_iterations; /* PBFluids.cpp:98 */
    p->max_lod = c->enable_apbf ? c->max_lod : c->solver_iterations; /* PBFluids.cpp:99 */
    p->lod_max_dist = c->lod_max_dist;
    p->iterations = c->solver_iterations;
}

/* getGridHash: int wrap-around products XORed, masked (CS_PredictAndHash.glsl:77-83). */
uint32_t orc_hash(int32_t cx, int32_t cy, int32_t cz, uint32_t mask)
{
    const uint32_t n = ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u);
    return n & mask;
}

static inline void cell_of(const orc_real* x, orc_real h, int32_t c[3])
{
    for (int a = 0; a < 3; ++a) c[a] = (int32_t)floor(x[a] / h);
}

void orc_keys_f32(const float* x4, uint32_t n, float h, uint32_t mask, uint32_t* keys)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const float* x = x4 + 4 * i;
        /* FP32 division then floor, as `ivec3(floor(predPos / ubo.h))` */
        const int32_t cx = (int32_t)floorf(x[0] / h);
        const int32_t cy = (int32_t)floorf(x[1] / h);
        const int32_t cz = (int32_t)floorf(x[2] / h);
        keys[i] = orc_hash(cx, cy, cz, mask);
    }
}

/* Stable counting sort by key: ties keep input (id) order, which is what an
 * LSD radix sort of (key, id) pairs with ids in identity order produces
 * (CS_RadixScatter.glsl:54-78 ranks by lid, buckets scanned column-major). */
void orc_stable_sort(const uint32_t* keys, uint32_t n, uint32_t hash_size, uint32_t* sorted_keys,
                     uint32_t* sorted_ids)
{
    uint32_t* count = (uint32_t*)calloc((size_t)hash_size + 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) count[keys[i] + 1]++;
    for (uint32_t k = 0; k < hash_size; ++k) count[k + 1] += count[k];
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t dst = count[keys[i]]++;
        sorted_keys[dst] = keys[i];
        sorted_ids[dst] = i;
    }
    free(count);
}

/* CS_BuildOffsets.glsl:55-78 */
void orc_build_table(const uint32_t* sk, uint32_t n, uint32_t hash_size, int32_t* table)
{
    for (uint32_t k = 0; k < 2u * hash_size; ++k) table[k] = -1; /* clearMode (:58-61) */
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t k = sk[i];
        if (i == 0 || sk[i - 1] != k) table[2 * k] = (int32_t)i;              /* :68-70 */
        if (i == n - 1 || sk[i + 1] != k) table[2 * k + 1] = (int32_t)(i + 1); /* :73-75 */
    }
}

/* ---- SDF grid sampling ---------------------------------------------------- */
static inline orc_real texel(const orc_sdf* s, int x, int y, int z)
{
    x = x < 0 ? 0 : (x >= s->dims[0] ? s->dims[0] - 1 : x);
    y = y < 0 ? 0 : (y >= s->dims[1] ? s->dims[1] - 1 : y);
    z = z < 0 ? 0 : (z >= s->dims[2] ? s->dims[2] - 1 : z);
    return (orc_real)s->dist[((int64_t)x * s->dims[1] + y) * s->dims[2] + z];
}

/* texture(sdfTexture, ((p - o)/cell + 0.5)/dims) with GL_LINEAR and
 * CLAMP_TO_EDGE (CS_Integrate.glsl:86-89, src/opengl/Texture3D.cpp:25-32):
 * texel-space coordinate u = (p - o)/cell, texel i centred on integer i. */
orc_real orc_sdf_query(const orc_sdf* s, const orc_real p[3])
{
    orc_real u[3];
    int i0[3];
    orc_real a[3];
    for (int k = 0; k < 3; ++k) {
        u[k] = clampd((p[k] - s->origin[k]) / s->cell, 0.0, (orc_real)(s->dims[k] - 1));
        i0[k] = (int)floor(u[k]);
        a[k] = u[k] - i0[k];
    }
    orc_real c[2][2][2];
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy)
            for (int dz = 0; dz < 2; ++dz) c[dx][dy][dz] = texel(s, i0[0] + dx, i0[1] + dy, i0[2] + dz);
    orc_real cz[2][2];
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy) cz[dx][dy] = c[dx][dy][0] + (c[dx][dy][1] - c[dx][dy][0]) * a[2];
    orc_real cy[2];
    for (int dx = 0; dx < 2; ++dx) cy[dx] = cz[dx][0] + (cz[dx][1] - cz[dx][0]) * a[1];
    return cy[0] + (cy[1] - cy[0]) * a[0];
}

/* sdfGradient: central differences with e = cell (CS_Integrate.glsl:92-99) */
void orc_sdf_gradient(const orc_sdf* s, const orc_real p[3], orc_real g[3])
{
    const orc_real e = s->cell;
    for (int k = 0; k < 3; ++k) {
        orc_real pp[3] = {p[0], p[1], p[2]}, pm[3] = {p[0], p[1], p[2]};
        pp[k] += e;
        pm[k] -= e;
        g[k] = (orc_sdf_query(s, pp) - orc_sdf_query(s, pm)) / (2.0 * e);
    }
}

/* ---- kernels (CS_ComputeLambdas.glsl:74-92) ------------------------------ */
static inline orc_real poly6(const orc_params* p, orc_real r2)
{
    if (r2 > p->h2) return 0.0;
    const orc_real d = p->h2 - r2;
    return p->poly6 * d * d * d;
}

static inline void grad_spiky(const orc_params* p, const orc_real r[3], orc_real r2, orc_real g[3])
{
    if (r2 > p->h2 || r2 < 1e-10) {
        g[0] = g[1] = g[2] = 0.0;
        return;
    }
    const orc_real dist = sqrt(r2);
    const orc_real diff = p->h - dist;
    const orc_real sc = -p->spiky * diff * diff / dist;
    g[0] = r[0] * sc;
    g[1] = r[1] * sc;
    g[2] = r[2] * sc;
}

/* computeSCorr (CS_ComputeDeltaP.glsl:94-104) */
static inline orc_real scorr(const orc_params* p, orc_real r2)
{
    if (!p->scorr) return 0.0;
    const orc_real w = poly6(p, r2);
    if (p->wq <= 1e-12 || w <= 0.0) return 0.0;
    const orc_real ratio = w / p->wq;
    if (ratio <= 0.0) return 0.0;
    return -p->k_corr * pow(ratio, p->n_corr);
}

/* ---- passes -------------------------------------------------------------- */
void orc_predict(const orc_params* p, uint32_t n, const orc_real* pos, orc_real* vel, orc_real* xstar,
                 uint32_t* keys)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_real* x = pos + 3 * i;
        orc_real* v = vel + 3 * i;
        for (int a = 0; a < 3; ++a) v[a] += p->g[a] * p->dt; /* :102 */
        if (p->interacting) {                                 /* :105-112 */
            orc_real to[3] = {p->i_pos[0] - x[0], p->i_pos[1] - x[1], p->i_pos[2] - x[2]};
            const orc_real dist = sqrt(dot3(to, to));
            if (dist < p->i_radius && dist > 1e-5) {
                const orc_real falloff = 1.0 - dist / p->i_radius;
                for (int a = 0; a < 3; ++a) v[a] += to[a] / dist * p->i_strength * falloff * p->dt;
            }
        }
        orc_real* xs = xstar + 3 * i;
        for (int a = 0; a < 3; ++a) xs[a] = x[a] + v[a] * p->dt; /* :114 */
        int32_t c[3];
        cell_of(xs, p->h, c); /* :125 */
        if (keys) keys[i] = orc_hash(c[0], c[1], c[2], p->mask);
    }
}

void orc_lod(const orc_params* p, uint32_t n, const orc_real* xstar, uint32_t* lod)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_real* x = xstar + 3 * i;
        orc_real d[3] = {p->camera[0] - x[0], p->camera[1] - x[1], p->camera[2] - x[2]};
        const orc_real dist = sqrt(dot3(d, d));
        const orc_real t = clampd(dist / p->lod_max_dist, 0.0, 1.0);
        const orc_real m = (orc_real)p->max_lod * (1.0 - t) + (orc_real)p->min_lod * t;
        uint32_t l = (uint32_t)rint(m);
        if (l < p->min_lod) l = p->min_lod;
        if (l > p->max_lod) l = p->max_lod;
        lod[i] = l;
    }
}

/* The 27-bucket loop shared by every neighbour shader: z outer, x inner
 * (CS_ComputeLambdas.glsl:126-150). */
#define FOR_EACH_NEIGHBOUR(p, xi, i, ids, table, ...)                                      \
    do {                                                                                     \
        int32_t c_[3];                                                                      \
        cell_of((xi), (p)->h, c_);                                                          \
        for (int z_ = -1; z_ <= 1; ++z_)                                                    \
            for (int y_ = -1; y_ <= 1; ++y_)                                                \
                for (int x_ = -1; x_ <= 1; ++x_) {                                          \
                    const uint32_t hh_ = orc_hash(c_[0] + x_, c_[1] + y_, c_[2] + z_, (p)->mask); \
                    const int32_t s_ = (table)[2 * hh_], e_ = (table)[2 * hh_ + 1];         \
                    if (s_ == -1) continue;                                                  \
                    for (int32_t k_ = s_; k_ < e_; ++k_) {                                   \
                        const uint32_t j = (ids)[k_];                                        \
                        if ((uint32_t)(i) == j) continue;                                    \
                        __VA_ARGS__                                                          \
                    }                                                                        \
                }                                                                            \
    } while (0)

void orc_lambda(const orc_params* p, uint32_t n, const orc_real* xstar, const uint32_t* ids,
                const int32_t* table, const uint32_t* lod, uint32_t iter, orc_real* lambda, orc_real* rho)
{
    const orc_real ir2 = p->inv_rho0 * p->inv_rho0;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        if (p->apbf && lod && lod[i] < iter) continue; /* :113 */
        const orc_real* xi = xstar + 3 * i;
        orc_real rho_i = p->w0_self, sg = 0.0, gi[3] = {0, 0, 0};
        FOR_EACH_NEIGHBOUR(p, xi, i, ids, table, {
            const orc_real* xj = xstar + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            rho_i += poly6(p, r2); /* :140 */
            orc_real g[3];
            grad_spiky(p, r, r2, g);
            sg += dot3(g, g) * ir2; /* :142-144 */
            gi[0] += g[0];
            gi[1] += g[1];
            gi[2] += g[2];
        });
        for (int a = 0; a < 3; ++a) gi[a] *= p->inv_rho0; /* :155 */
        orc_real C = rho_i / p->rho0 - 1.0;
        if (C < -p->cohesion) C = -p->cohesion; /* :156 */
        sg += dot3(gi, gi);                      /* :157 */
        lambda[i] = -C / (sg + p->eps);          /* :158 */
        if (rho) rho[i] = rho_i;
    }
}

/* Obstacle / container projection (CS_ApplyDeltaP.glsl:108-121,
 * CS_Integrate.glsl:216-240).  Returns 1 and the push normal on contact. */
static int sdf_project(const orc_sdf* s, orc_real x[3], orc_real nrm[3])
{
    const orc_real d = orc_sdf_query(s, x);
    orc_real g[3];
    orc_sdf_gradient(s, x, g);
    const orc_real len = sqrt(dot3(g, g));
    if (!(len > 1e-6)) return 0;
    if (s->containment) {
        if (d > -s->padding) {
            for (int a = 0; a < 3; ++a) {
                nrm[a] = -g[a] / len;
                x[a] += nrm[a] * (d + s->padding);
            }
            return 1;
        }
    } else {
        if (d < s->padding) {
            for (int a = 0; a < 3; ++a) {
                nrm[a] = g[a] / len;
                x[a] += nrm[a] * (s->padding - d);
            }
            return 1;
        }
    }
    return 0;
}

void orc_deltap_apply(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* xstar,
                      const orc_real* lambda, const uint32_t* ids, const int32_t* table,
                      const uint32_t* lod, uint32_t iter, orc_real* dp_out)
{
    orc_real* dp = dp_out ? dp_out : (orc_real*)malloc(sizeof(orc_real) * 3 * (size_t)n);
    /* CS_ComputeDeltaP.glsl:120-166 */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        if (p->apbf && lod && lod[i] < iter) continue; /* :125 */
        const orc_real* xi = xstar + 3 * i;
        const orc_real li = lambda[i];
        orc_real acc[3] = {0, 0, 0};
        FOR_EACH_NEIGHBOUR(p, xi, i, ids, table, {
            const orc_real* xj = xstar + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            orc_real g[3];
            grad_spiky(p, r, r2, g);
            const orc_real f = li + lambda[j] + scorr(p, r2); /* :155-156 */
            acc[0] += g[0] * f;
            acc[1] += g[1] * f;
            acc[2] += g[2] * f;
        });
        for (int a = 0; a < 3; ++a) dp[3 * i + a] = acc[a] * p->inv_rho0; /* :165 */
    }
    /* CS_ApplyDeltaP.glsl:80-124 */
    const orc_real maxdp = 0.5 * p->h;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        if (p->apbf && lod && lod[i] < iter) continue; /* :85 */
        orc_real d[3] = {dp[3 * i], dp[3 * i + 1], dp[3 * i + 2]};
        const orc_real l2 = dot3(d, d);
        if (l2 > maxdp * maxdp) { /* :92-100 */
            const orc_real sc = maxdp / sqrt(l2);
            d[0] *= sc;
            d[1] *= sc;
            d[2] *= sc;
        }
        orc_real x[3] = {xstar[3 * i] + d[0], xstar[3 * i + 1] + d[1], xstar[3 * i + 2] + d[2]};
        if (s && s->enabled) {
            orc_real nrm[3];
            sdf_project(s, x, nrm);
        }
        xstar[3 * i] = x[0];
        xstar[3 * i + 1] = x[1];
        xstar[3 * i + 2] = x[2];
    }
    if (!dp_out) free(dp);
}

void orc_integrate(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* pos, orc_real* vel,
                   const orc_real* xstar, const uint32_t* ids, const int32_t* table, orc_real* omega)
{
    /* neighbour velocities are read from before the dispatch */
    orc_real* v0 = (orc_real*)malloc(sizeof(orc_real) * 3 * (size_t)n);
    memcpy(v0, vel, sizeof(orc_real) * 3 * (size_t)n);
    const orc_real inv_dt = (p->dt > 0.0) ? 1.0 / p->dt : 0.0; /* :244 */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_real* old_pos = pos + 3 * i;
        const orc_real* old_vel = v0 + 3 * i;
        orc_real x[3] = {xstar[3 * i], xstar[3 * i + 1], xstar[3 * i + 2]};
        orc_real visc_delta[3] = {0, 0, 0};
        if (p->visc_on || p->vort_on) { /* :153-194 */
            orc_real vf[3] = {0, 0, 0}, curl[3] = {0, 0, 0};
            FOR_EACH_NEIGHBOUR(p, x, i, ids, table, {
                const orc_real* xj = xstar + 3 * j;
                const orc_real* vj = v0 + 3 * j;
                const orc_real r[3] = {x[0] - xj[0], x[1] - xj[1], x[2] - xj[2]};
                const orc_real r2 = dot3(r, r);
                const orc_real vij[3] = {vj[0] - old_vel[0], vj[1] - old_vel[1], vj[2] - old_vel[2]};
                if (p->visc_on) {
                    const orc_real w = poly6(p, r2);
                    for (int a = 0; a < 3; ++a) vf[a] += vij[a] * w * p->inv_rho0; /* :177 */
                }
                if (p->vort_on) {
                    orc_real g[3];
                    grad_spiky(p, r, r2, g);
                    curl[0] += vij[1] * g[2] - vij[2] * g[1]; /* :182 */
                    curl[1] += vij[2] * g[0] - vij[0] * g[2];
                    curl[2] += vij[0] * g[1] - vij[1] * g[0];
                }
            });
            if (p->visc_on)
                for (int a = 0; a < 3; ++a) visc_delta[a] = vf[a] * p->viscosity; /* :192 */
            if (p->vort_on && omega)
                for (int a = 0; a < 3; ++a) omega[3 * i + a] = curl[a] * p->inv_rho0; /* :193 */
        }
        int col[3] = {0, 0, 0}; /* :199-210 */
        for (int a = 0; a < 3; ++a) {
            if (x[a] <= p->bmin[a]) { x[a] = p->bmin[a]; col[a] = 1; }
            if (x[a] >= p->bmax[a]) { x[a] = p->bmax[a]; col[a] = 1; }
        }
        int col_sdf = 0;
        orc_real nrm[3] = {0, 0, 0};
        if (s && s->enabled) col_sdf = sdf_project(s, x, nrm); /* :216-240 */
        orc_real v[3];
        for (int a = 0; a < 3; ++a) v[a] = (x[a] - old_pos[a]) * inv_dt + visc_delta[a]; /* :246,252 */
        const orc_real sp2 = dot3(v, v);
        if (sp2 > 2500.0) { /* :255-256 */
            const orc_real sc = 50.0 / sqrt(sp2);
            for (int a = 0; a < 3; ++a) v[a] *= sc;
        }
        for (int a = 0; a < 3; ++a)
            if (col[a]) v[a] *= -p->damping; /* :259-261 */
        if (col_sdf) {                       /* :268-271 */
            const orc_real vn = dot3(v, nrm);
            for (int a = 0; a < 3; ++a) v[a] -= vn * nrm[a];
        }
        for (int a = 0; a < 3; ++a) { /* :276-277 */
            pos[3 * i + a] = x[a];
            vel[3 * i + a] = v[a];
        }
    }
    free(v0);
}

void orc_vorticity(const orc_params* p, uint32_t n, const orc_real* pos, orc_real* vel,
                   const orc_real* omega, const uint32_t* ids, const int32_t* table)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_real* xi = pos + 3 * i;
        orc_real eta[3] = {0, 0, 0};
        FOR_EACH_NEIGHBOUR(p, xi, i, ids, table, { /* :139-155 */
            const orc_real* xj = pos + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            orc_real g[3];
            grad_spiky(p, r, r2, g);
            const orc_real om = sqrt(dot3(omega + 3 * j, omega + 3 * j));
            eta[0] += om * g[0];
            eta[1] += om * g[1];
            eta[2] += om * g[2];
        });
        for (int a = 0; a < 3; ++a) eta[a] *= p->inv_rho0; /* :157 */
        const orc_real el = sqrt(dot3(eta, eta));
        if (el < 1e-6) continue; /* :160 */
        const orc_real N[3] = {eta[0] / el, eta[1] / el, eta[2] / el};
        const orc_real* w = omega + 3 * i;
        const orc_real cr[3] = {N[1] * w[2] - N[2] * w[1], N[2] * w[0] - N[0] * w[2], N[0] * w[1] - N[1] * w[0]};
        for (int a = 0; a < 3; ++a) vel[3 * i + a] += p->vort_eps * cr[a] * p->dt; /* :166 */
    }
}

void orc_step(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* pos, orc_real* vel,
              orc_real* omega, orc_real* rho, uint32_t* sorted_keys_out, uint32_t* sorted_ids_out,
              int32_t* table_out)
{
    if (n == 0) return; /* PBFluids.cpp:325 */
    const uint32_t H = p->hash_size;
    orc_real* xs = (orc_real*)malloc(sizeof(orc_real) * 3 * (size_t)n);
    orc_real* lam = (orc_real*)calloc((size_t)n, sizeof(orc_real));
    orc_real* rh = (orc_real*)malloc(sizeof(orc_real) * (size_t)n);
    orc_real* om = (orc_real*)calloc(3 * (size_t)n, sizeof(orc_real));
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t* sk = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t* ids = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    int32_t* table = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)H);
    uint32_t* lod = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    for (uint32_t i = 0; i < n; ++i) { lod[i] = p->apbf ? p->max_lod : p->iterations; rh[i] = 0.0; }
    const uint32_t max_iter = p->apbf ? p->max_lod : p->iterations; /* :455 */

    for (uint32_t sub = 0; sub < p->substeps; ++sub) { /* :344 */
        orc_predict(p, n, pos, vel, xs, keys);          /* :347-349 */
        memset(lam, 0, sizeof(orc_real) * (size_t)n);     /* CS_PredictAndHash.glsl:121 */
        orc_stable_sort(keys, n, H, sk, ids);           /* :354-405 */
        orc_build_table(sk, n, H, table);               /* :408-418 */
        if (p->apbf) orc_lod(p, n, xs, lod);            /* :421-426 */
        for (uint32_t it = 1; it <= max_iter; ++it) {   /* :456-472 */
            orc_lambda(p, n, xs, ids, table, lod, it, lam, rh);
            orc_deltap_apply(p, s, n, xs, lam, ids, table, lod, it, NULL);
        }
        orc_integrate(p, s, n, pos, vel, xs, ids, table, om); /* :475-495 */
    }
    if (p->vort_on) orc_vorticity(p, n, pos, vel, om, ids, table); /* :499-505 */

    if (omega) memcpy(omega, om, sizeof(orc_real) * 3 * (size_t)n);
    if (rho) memcpy(rho, rh, sizeof(orc_real) * (size_t)n);
    if (sorted_keys_out) memcpy(sorted_keys_out, sk, sizeof(uint32_t) * (size_t)n);
    if (sorted_ids_out) memcpy(sorted_ids_out, ids, sizeof(uint32_t) * (size_t)n);
    if (table_out) memcpy(table_out, table, sizeof(int32_t) * 2 * (size_t)H);
    free(xs); free(lam); free(rh); free(om); free(keys); free(sk); free(ids); free(table); free(lod);
}

/* CS_ContactFilter.glsl:68-83 */
uint32_t orc_contact_filter(const orc_sdf* s, uint32_t n, const orc_real* pos, orc_real band,
                            uint32_t* out_idx)
{
    if (!s || !s->enabled || band <= 0.0) return 0; /* PBFluids.cpp:195 */
    uint32_t c = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const orc_real d = orc_sdf_query(s, pos + 3 * i);
        if (fabs(d) < band) out_idx[c++] = i;
    }
    return c;
}

/* Kernel values for pinning against src/fluid/Kernels.cpp:9-27,116-141. */
void orc_kernels(const orc_params* p, const orc_real r[3], orc_real* w, orc_real g[3])
{
    const orc_real r2 = dot3(r, r);
    *w = poly6(p, r2);
    grad_spiky(p, r, r2, g);
}

/* Visited candidates within h (r^2 <= h^2, with bucket multiplicity) — the
 * neighbour lists NeighborSearch::build (src/fluid/NeighborSearch.cpp:97-126)
 * produces when its cell size equals h. */
void orc_neighbor_lists(const orc_params* p, uint32_t n, const orc_real* x, const uint32_t* ids,
                        const int32_t* table, int32_t* counts, int32_t* lists, int32_t cap)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_real* xi = x + 3 * i;
        int32_t c = 0;
        FOR_EACH_NEIGHBOUR(p, xi, i, ids, table, {
            const orc_real* xj = x + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            if (dot3(r, r) <= p->h2) {
                if (lists && c < cap) lists[i * cap + c] = (int32_t)j;
                ++c;
            }
        });
        counts[i] = c;
    }
}
