/*
 * pbf_adjoint.c — FP64 reverse-mode derivative of the oracle's PBF step.
 *
 * TEST INFRASTRUCTURE ONLY (see pbf_oracle.h): the CPU reference gradient the
 * GPU adjoint kernels are checked against, itself checked against FP64
 * central differences of orc_step.
 *
 * The forward is orc_step (PBFluids::step, src/fluid/PBFluids.cpp:323-517)
 * with the SDF translated by t (grid origin + t).  Discrete choices — the
 * sort permutation, the neighbour sets, wall and SDF contacts, the Δp and
 * speed clamps, the cohesion clamp — are replayed from the recomputed
 * forward and differentiated as the constant branches they are on each side.
 * Per substep the state at the substep start is checkpointed; the backward
 * recomputes the substep from its checkpoint (predict, sort, table, every
 * solver iteration) and then runs, in reverse: vorticity (last substep),
 * integrate, (deltaP+apply, lambda) for each iteration, predict.  Pair terms
 * are scattered to the neighbour with atomic adds.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pbf_oracle.h"

static inline orc_real dot3(const orc_real* a, const orc_real* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* poly6 value and d/d(r^2) (CS_ComputeLambdas.glsl:74-81), r2 <= h2 */
static inline orc_real poly6_v(const orc_params* p, orc_real r2) { orc_real d = p->h2 - r2; return p->poly6 * d * d * d; }
static inline orc_real poly6_d(const orc_params* p, orc_real r2) { orc_real d = p->h2 - r2; return -3.0 * p->poly6 * d * d; }
/* spiky gradient factor s (grad = r s) and ds/d(r^2), 1e-10 <= r2 <= h2
 * (CS_ComputeLambdas.glsl:83-92) */
static inline orc_real spiky_s(const orc_params* p, orc_real r2)
{
    const orc_real q = sqrt(r2), d = p->h - q;
    return -p->spiky * d * d / q;
}
static inline orc_real spiky_ds(const orc_params* p, orc_real r2)
{
    const orc_real q = sqrt(r2);
    return p->spiky * (p->h - q) * (p->h + q) / (2.0 * q * q * q);
}
/* s_corr and d/d(r^2) (CS_ComputeDeltaP.glsl:94-104), r2 <= h2 */
static inline orc_real scorr_v(const orc_params* p, orc_real r2)
{
    if (!p->scorr) return 0.0;
    const orc_real w = poly6_v(p, r2);
    if (p->wq <= 1e-12 || w <= 0.0) return 0.0;
    return -p->k_corr * pow(w / p->wq, p->n_corr);
}
static inline orc_real scorr_d(const orc_params* p, orc_real r2)
{
    if (!p->scorr) return 0.0;
    const orc_real w = poly6_v(p, r2);
    if (p->wq <= 1e-12 || w <= 0.0) return 0.0;
    return -p->k_corr * p->n_corr * pow(w / p->wq, p->n_corr - 1.0) / p->wq * poly6_d(p, r2);
}

/* adjoint of a = r s(r^2) given a_bar: r_bar += s a_bar + 2 ds (r . a_bar) r */
static inline void grad_vjp(const orc_params* p, const orc_real r[3], orc_real r2, const orc_real ab[3], orc_real rb[3])
{
    const orc_real s = spiky_s(p, r2), ds = spiky_ds(p, r2), k = 2.0 * ds * dot3(r, ab);
    for (int a = 0; a < 3; ++a) rb[a] += s * ab[a] + k * r[a];
}

static inline void atomic_sub3(orc_real* dst, const orc_real v[3])
{
    for (int a = 0; a < 3; ++a) {
#pragma omp atomic
        dst[a] -= v[a];
    }
}

static inline void atomic_add1(orc_real* dst, orc_real v)
{
#pragma omp atomic
    *dst += v;
}

/* the 27-bucket walk (CS_ComputeLambdas.glsl:126-150): j over every visit */
#define ADJ_FOR_EACH(p, xi, i, ids, table, ...)                                                    \
    do {                                                                                            \
        int32_t c_[3];                                                                              \
        for (int a_ = 0; a_ < 3; ++a_) c_[a_] = (int32_t)floor((xi)[a_] / (p)->h);                  \
        for (int z_ = -1; z_ <= 1; ++z_)                                                            \
            for (int y_ = -1; y_ <= 1; ++y_)                                                        \
                for (int x_ = -1; x_ <= 1; ++x_) {                                                  \
                    const uint32_t hh_ = orc_hash(c_[0] + x_, c_[1] + y_, c_[2] + z_, (p)->mask);   \
                    const int32_t s_ = (table)[2 * hh_], e_ = (table)[2 * hh_ + 1];                 \
                    if (s_ == -1) continue;                                                          \
                    for (int32_t k_ = s_; k_ < e_; ++k_) {                                           \
                        const uint32_t j = (ids)[k_];                                                \
                        if ((uint32_t)(i) == j) continue;                                            \
                        __VA_ARGS__                                                                  \
                    }                                                                                \
                }                                                                                    \
    } while (0)

/* ---- SDF: value, analytic gradient of the trilinear interpolant ---------- */
static inline orc_real texel(const orc_sdf* s, int x, int y, int z)
{
    x = x < 0 ? 0 : (x >= s->dims[0] ? s->dims[0] - 1 : x);
    y = y < 0 ? 0 : (y >= s->dims[1] ? s->dims[1] - 1 : y);
    z = z < 0 ? 0 : (z >= s->dims[2] ? s->dims[2] - 1 : z);
    return (orc_real)s->dist[((int64_t)x * s->dims[1] + y) * s->dims[2] + z];
}

/* d orc_sdf_query / dp (zero along an axis where the coordinate is clamped) */
static orc_real sdf_grad_exact(const orc_sdf* s, const orc_real p[3], orc_real gr[3])
{
    orc_real a[3];
    int i0[3], live[3];
    for (int k = 0; k < 3; ++k) {
        const orc_real u = (p[k] - s->origin[k]) / s->cell;
        const orc_real hi = (orc_real)(s->dims[k] - 1);
        live[k] = (u > 0.0 && u < hi);
        const orc_real uc = u < 0.0 ? 0.0 : (u > hi ? hi : u);
        i0[k] = (int)floor(uc);
        a[k] = uc - i0[k];
    }
    orc_real c[2][2][2];
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy)
            for (int dz = 0; dz < 2; ++dz) c[dx][dy][dz] = texel(s, i0[0] + dx, i0[1] + dy, i0[2] + dz);
    const orc_real w0[2] = {1.0 - a[0], a[0]}, w1[2] = {1.0 - a[1], a[1]};
    orc_real cz[2][2], dz_[2][2];
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy) {
            cz[dx][dy] = c[dx][dy][0] + (c[dx][dy][1] - c[dx][dy][0]) * a[2];
            dz_[dx][dy] = c[dx][dy][1] - c[dx][dy][0];
        }
    orc_real cy[2];
    for (int dx = 0; dx < 2; ++dx) cy[dx] = cz[dx][0] + (cz[dx][1] - cz[dx][0]) * a[1];
    const orc_real val = cy[0] + (cy[1] - cy[0]) * a[0];
    const orc_real d0 = cy[1] - cy[0];
    const orc_real d1 = w0[0] * (cz[0][1] - cz[0][0]) + w0[1] * (cz[1][1] - cz[1][0]);
    orc_real d2 = 0.0;
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy) d2 += w0[dx] * w1[dy] * dz_[dx][dy];
    const orc_real inv = 1.0 / s->cell;
    gr[0] = live[0] ? d0 * inv : 0.0;
    gr[1] = live[1] ? d1 * inv : 0.0;
    gr[2] = live[2] ? d2 * inv : 0.0;
    return val;
}

/* Vector-Jacobian product of the obstacle/container projection
 * (CS_ApplyDeltaP.glsl:108-121, CS_Integrate.glsl:216-240) at input point x:
 * xb (adjoint of the projected point) is replaced by the adjoint of x, nb is
 * the adjoint of the returned push normal; tb += adjoint of the translation.
 * Returns 1 when x was projected. */
static int project_vjp(const orc_sdf* s, const orc_real x[3], orc_real xb[3], const orc_real nb[3], orc_real tb[3])
{
    const orc_real e = s->cell;
    orc_real gq[3];
    const orc_real d = sdf_grad_exact(s, x, gq);
    orc_real G[3], H[3][3];
    for (int k = 0; k < 3; ++k) {
        orc_real pp[3] = {x[0], x[1], x[2]}, pm[3] = {x[0], x[1], x[2]};
        pp[k] += e;
        pm[k] -= e;
        orc_real gp[3], gm[3];
        const orc_real vp = sdf_grad_exact(s, pp, gp), vm = sdf_grad_exact(s, pm, gm);
        G[k] = (vp - vm) / (2.0 * e);
        for (int m = 0; m < 3; ++m) H[k][m] = (gp[m] - gm[m]) / (2.0 * e);
    }
    const orc_real len = sqrt(dot3(G, G));
    if (!(len > 1e-6)) return 0;
    orc_real n[3], sc;
    if (s->containment) {
        if (!(d > -s->padding)) return 0;
        for (int a = 0; a < 3; ++a) n[a] = -G[a] / len;
        sc = d + s->padding;
    } else {
        if (!(d < s->padding)) return 0;
        for (int a = 0; a < 3; ++a) n[a] = G[a] / len;
        sc = s->padding - d;
    }
    /* x' = x + n sc.  dn/dx = sgn (I - n n^T) H / len with sgn = -1 in
     * containment; dsc/dx = -+grad q. */
    const orc_real sgn = s->containment ? -1.0 : 1.0;
    /* v = sc * xb + nb  -> contribution H^T (I - n n^T) v sgn / len */
    orc_real v[3];
    for (int a = 0; a < 3; ++a) v[a] = sc * xb[a] + nb[a];
    const orc_real nv = dot3(n, v);
    orc_real pv[3];
    for (int a = 0; a < 3; ++a) pv[a] = (v[a] - n[a] * nv) * sgn / len;
    orc_real add[3] = {0, 0, 0};
    for (int m = 0; m < 3; ++m)
        for (int k = 0; k < 3; ++k) add[m] += H[k][m] * pv[k];
    const orc_real nxb = dot3(n, xb);
    for (int a = 0; a < 3; ++a) add[a] += (s->containment ? 1.0 : -1.0) * gq[a] * nxb;
    for (int a = 0; a < 3; ++a) {
        xb[a] += add[a];
        if (tb) tb[a] -= add[a];
    }
    return 1;
}

/* ---- per-pass adjoints ----------------------------------------------------- */
/* CS_ComputeLambdas.glsl:108-162 reversed: lamb -> xsb (accumulated) */
static void lambda_vjp(const orc_params* p, uint32_t n, const orc_real* xs, const uint32_t* ids, const int32_t* table,
                       const orc_real* lamb, orc_real* xsb)
{
    const orc_real ir2 = p->inv_rho0 * p->inv_rho0;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        if (lamb[i] == 0.0) continue;
        const orc_real* xi = xs + 3 * i;
        orc_real rho = p->w0_self, sg = 0.0, gs[3] = {0, 0, 0};
        ADJ_FOR_EACH(p, xi, i, ids, table, {
            const orc_real* xj = xs + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            if (r2 <= p->h2) {
                rho += poly6_v(p, r2);
                if (r2 >= 1e-10) {
                    const orc_real s = spiky_s(p, r2);
                    sg += s * s * r2 * ir2;
                    for (int a = 0; a < 3; ++a) gs[a] += r[a] * s;
                }
            }
        });
        orc_real gi[3] = {gs[0] * p->inv_rho0, gs[1] * p->inv_rho0, gs[2] * p->inv_rho0};
        const orc_real craw = rho / p->rho0 - 1.0;
        const orc_real C = craw < -p->cohesion ? -p->cohesion : craw;
        const orc_real D = sg + dot3(gi, gi) + p->eps;
        const orc_real Cb = -lamb[i] / D;
        const orc_real Db = lamb[i] * C / (D * D);
        const orc_real rhob = (craw < -p->cohesion) ? 0.0 : Cb / p->rho0;
        orc_real gsb[3];
        for (int a = 0; a < 3; ++a) gsb[a] = Db * 2.0 * gi[a] * p->inv_rho0;
        orc_real own[3] = {0, 0, 0};
        ADJ_FOR_EACH(p, xi, i, ids, table, {
            const orc_real* xj = xs + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            if (r2 <= p->h2) {
                orc_real rb[3] = {0, 0, 0};
                const orc_real k = rhob * poly6_d(p, r2) * 2.0;
                for (int a = 0; a < 3; ++a) rb[a] += k * r[a];
                if (r2 >= 1e-10) {
                    const orc_real s = spiky_s(p, r2);
                    orc_real ab[3];
                    for (int a = 0; a < 3; ++a) ab[a] = Db * 2.0 * r[a] * s * ir2 + gsb[a];
                    grad_vjp(p, r, r2, ab, rb);
                }
                for (int a = 0; a < 3; ++a) own[a] += rb[a];
                atomic_sub3(xsb + 3 * j, rb);
            }
        });
        for (int a = 0; a < 3; ++a) atomic_add1(xsb + 3 * i + a, own[a]);
    }
}

/* CS_ComputeDeltaP.glsl:120-166 + CS_ApplyDeltaP.glsl:80-124 reversed:
 * xsb_out (adjoint of the output x*) -> xsb_prev, lamb (accumulated) */
static void deltap_vjp(const orc_params* p, const orc_sdf* s, uint32_t n, const orc_real* xs, const orc_real* lam,
                       const uint32_t* ids, const int32_t* table, const orc_real* xsb_out, orc_real* xsb_prev,
                       orc_real* lamb, orc_real* tb)
{
    const orc_real maxdp = 0.5 * p->h;
    orc_real tacc[3] = {0, 0, 0};
#pragma omp parallel
    {
        orc_real tloc[3] = {0, 0, 0};
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            const orc_real* xi = xs + 3 * i;
            const orc_real li = lam[i];
            orc_real acc[3] = {0, 0, 0};
            ADJ_FOR_EACH(p, xi, i, ids, table, {
                const orc_real* xj = xs + 3 * j;
                const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
                const orc_real r2 = dot3(r, r);
                if (r2 <= p->h2 && r2 >= 1e-10) {
                    const orc_real sc = spiky_s(p, r2) * (li + lam[j] + scorr_v(p, r2));
                    for (int a = 0; a < 3; ++a) acc[a] += r[a] * sc;
                }
            });
            orc_real dp[3] = {acc[0] * p->inv_rho0, acc[1] * p->inv_rho0, acc[2] * p->inv_rho0};
            const orc_real l2 = dot3(dp, dp);
            const int clamped = l2 > maxdp * maxdp;
            orc_real dpc[3] = {dp[0], dp[1], dp[2]};
            if (clamped) {
                const orc_real k = maxdp / sqrt(l2);
                for (int a = 0; a < 3; ++a) dpc[a] *= k;
            }
            orc_real x[3] = {xi[0] + dpc[0], xi[1] + dpc[1], xi[2] + dpc[2]};
            orc_real xb[3] = {xsb_out[3 * i], xsb_out[3 * i + 1], xsb_out[3 * i + 2]};
            if (s && s->enabled) {
                const orc_real zero[3] = {0, 0, 0};
                project_vjp(s, x, xb, zero, tloc);
            }
            orc_real dpb[3] = {xb[0], xb[1], xb[2]};
            if (clamped) {
                const orc_real len = sqrt(l2);
                orc_real u[3] = {dp[0] / len, dp[1] / len, dp[2] / len};
                const orc_real ub = dot3(u, xb);
                for (int a = 0; a < 3; ++a) dpb[a] = maxdp / len * (xb[a] - u[a] * ub);
            }
            orc_real accb[3] = {dpb[0] * p->inv_rho0, dpb[1] * p->inv_rho0, dpb[2] * p->inv_rho0};
            orc_real own[3] = {xb[0], xb[1], xb[2]};
            orc_real lown = 0.0;
            ADJ_FOR_EACH(p, xi, i, ids, table, {
                const orc_real* xj = xs + 3 * j;
                const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
                const orc_real r2 = dot3(r, r);
                if (r2 <= p->h2 && r2 >= 1e-10) {
                    const orc_real s_ = spiky_s(p, r2);
                    const orc_real f = li + lam[j] + scorr_v(p, r2);
                    const orc_real ga = s_ * dot3(r, accb); /* grad . acc_bar */
                    lown += ga;
                    atomic_add1(lamb + j, ga);
                    orc_real rb[3] = {0, 0, 0};
                    orc_real ab[3] = {f * accb[0], f * accb[1], f * accb[2]};
                    grad_vjp(p, r, r2, ab, rb);
                    const orc_real k = ga * scorr_d(p, r2) * 2.0;
                    for (int a = 0; a < 3; ++a) rb[a] += k * r[a];
                    for (int a = 0; a < 3; ++a) own[a] += rb[a];
                    atomic_sub3(xsb_prev + 3 * j, rb);
                }
            });
            atomic_add1(lamb + i, lown);
            for (int a = 0; a < 3; ++a) atomic_add1(xsb_prev + 3 * i + a, own[a]);
        }
        for (int a = 0; a < 3; ++a) atomic_add1(tacc + a, tloc[a]);
    }
    if (tb)
        for (int a = 0; a < 3; ++a) tb[a] += tacc[a];
}

/* CS_Integrate.glsl:135-280 reversed: (posb, velb, omb) of the committed
 * state -> xsb (adjoint of x*), vpb (of the predicted velocity), x0b (of the
 * substep start position), all accumulated. */
static void integrate_vjp(const orc_params* p, const orc_sdf* s, uint32_t n, const orc_real* xs, const orc_real* vp,
                          const orc_real* x0, const uint32_t* ids, const int32_t* table, const orc_real* posb,
                          const orc_real* velb, const orc_real* omb, orc_real* xsb, orc_real* vpb, orc_real* x0b, orc_real* tb)
{
    const orc_real inv_dt = (p->dt > 0.0) ? 1.0 / p->dt : 0.0;
    orc_real tacc[3] = {0, 0, 0};
#pragma omp parallel
    {
        orc_real tloc[3] = {0, 0, 0};
#pragma omp for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; ++i) {
            const orc_real* xi = xs + 3 * i;
            const orc_real* vi = vp + 3 * i;
            orc_real vf[3] = {0, 0, 0};
            if (p->visc_on) {
                ADJ_FOR_EACH(p, xi, i, ids, table, {
                    const orc_real* xj = xs + 3 * j;
                    const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
                    const orc_real r2 = dot3(r, r);
                    if (r2 <= p->h2) {
                        const orc_real w = poly6_v(p, r2) * p->inv_rho0;
                        for (int a = 0; a < 3; ++a) vf[a] += (vp[3 * j + a] - vi[a]) * w;
                    }
                });
            }
            orc_real x[3] = {xi[0], xi[1], xi[2]};
            int col[3] = {0, 0, 0};
            for (int a = 0; a < 3; ++a) {
                if (x[a] <= p->bmin[a]) { x[a] = p->bmin[a]; col[a] = 1; }
                if (x[a] >= p->bmax[a]) { x[a] = p->bmax[a]; col[a] = 1; }
            }
            const orc_real xw[3] = {x[0], x[1], x[2]};
            orc_real nrm[3] = {0, 0, 0};
            int col_sdf = 0;
            if (s && s->enabled) {
                /* forward projection (same as orc_integrate) to get the normal */
                orc_real g[3];
                const orc_real d = orc_sdf_query(s, x);
                orc_sdf_gradient(s, x, g);
                const orc_real len = sqrt(dot3(g, g));
                if (len > 1e-6) {
                    if (s->containment ? (d > -s->padding) : (d < s->padding)) {
                        const orc_real sg = s->containment ? -1.0 : 1.0;
                        const orc_real sc = s->containment ? (d + s->padding) : (s->padding - d);
                        for (int a = 0; a < 3; ++a) {
                            nrm[a] = sg * g[a] / len;
                            x[a] += nrm[a] * sc;
                        }
                        col_sdf = 1;
                    }
                }
            }
            orc_real v1[3];
            for (int a = 0; a < 3; ++a)
                v1[a] = (x[a] - x0[3 * i + a]) * inv_dt + (p->visc_on ? vf[a] * p->viscosity : 0.0);
            const orc_real sp2 = dot3(v1, v1);
            orc_real v2[3] = {v1[0], v1[1], v1[2]};
            if (sp2 > 2500.0) {
                const orc_real k = 50.0 / sqrt(sp2);
                for (int a = 0; a < 3; ++a) v2[a] *= k;
            }
            orc_real v3[3];
            for (int a = 0; a < 3; ++a) v3[a] = col[a] ? v2[a] * -p->damping : v2[a];
            /* backward */
            orc_real vb[3] = {velb ? velb[3 * i] : 0.0, velb ? velb[3 * i + 1] : 0.0, velb ? velb[3 * i + 2] : 0.0};
            orc_real nb[3] = {0, 0, 0};
            if (col_sdf) {
                const orc_real vn = dot3(v3, nrm), nvb = dot3(nrm, vb);
                for (int a = 0; a < 3; ++a) nb[a] = -(vn * vb[a] + nvb * v3[a]);
                for (int a = 0; a < 3; ++a) vb[a] -= nrm[a] * nvb;
            }
            for (int a = 0; a < 3; ++a)
                if (col[a]) vb[a] *= -p->damping;
            if (sp2 > 2500.0) {
                const orc_real len = sqrt(sp2);
                const orc_real u[3] = {v1[0] / len, v1[1] / len, v1[2] / len};
                const orc_real ub = dot3(u, vb);
                for (int a = 0; a < 3; ++a) vb[a] = 50.0 / len * (vb[a] - u[a] * ub);
            }
            orc_real xb[3];
            for (int a = 0; a < 3; ++a) {
                xb[a] = (posb ? posb[3 * i + a] : 0.0) + vb[a] * inv_dt;
                x0b[3 * i + a] -= vb[a] * inv_dt;
            }
            if (col_sdf) project_vjp(s, xw, xb, nb, tloc);
            orc_real own[3];
            for (int a = 0; a < 3; ++a) own[a] = col[a] ? 0.0 : xb[a];
            orc_real vfb[3] = {0, 0, 0}, cb[3] = {0, 0, 0};
            if (p->visc_on)
                for (int a = 0; a < 3; ++a) vfb[a] = vb[a] * p->viscosity;
            if (p->vort_on && omb)
                for (int a = 0; a < 3; ++a) cb[a] = omb[3 * i + a] * p->inv_rho0;
            orc_real vown[3] = {0, 0, 0};
            ADJ_FOR_EACH(p, xi, i, ids, table, {
                const orc_real* xj = xs + 3 * j;
                const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
                const orc_real r2 = dot3(r, r);
                if (r2 <= p->h2) {
                    const orc_real u[3] = {vp[3 * j] - vi[0], vp[3 * j + 1] - vi[1], vp[3 * j + 2] - vi[2]};
                    orc_real ub[3] = {0, 0, 0}, rb[3] = {0, 0, 0};
                    if (p->visc_on) {
                        const orc_real w = poly6_v(p, r2) * p->inv_rho0;
                        for (int a = 0; a < 3; ++a) ub[a] += vfb[a] * w;
                        const orc_real k = dot3(vfb, u) * p->inv_rho0 * poly6_d(p, r2) * 2.0;
                        for (int a = 0; a < 3; ++a) rb[a] += k * r[a];
                    }
                    if (p->vort_on && r2 >= 1e-10) {
                        const orc_real s_ = spiky_s(p, r2);
                        const orc_real g[3] = {r[0] * s_, r[1] * s_, r[2] * s_};
                        /* curl += u x g */
                        ub[0] += g[1] * cb[2] - g[2] * cb[1];
                        ub[1] += g[2] * cb[0] - g[0] * cb[2];
                        ub[2] += g[0] * cb[1] - g[1] * cb[0];
                        const orc_real gb[3] = {cb[1] * u[2] - cb[2] * u[1], cb[2] * u[0] - cb[0] * u[2],
                                              cb[0] * u[1] - cb[1] * u[0]};
                        grad_vjp(p, r, r2, gb, rb);
                    }
                    for (int a = 0; a < 3; ++a) {
                        own[a] += rb[a];
                        vown[a] -= ub[a];
                    }
                    for (int a = 0; a < 3; ++a) atomic_add1(vpb + 3 * j + a, ub[a]);
                    atomic_sub3(xsb + 3 * j, rb);
                }
            });
            for (int a = 0; a < 3; ++a) {
                atomic_add1(xsb + 3 * i + a, own[a]);
                atomic_add1(vpb + 3 * i + a, vown[a]);
            }
        }
        for (int a = 0; a < 3; ++a) atomic_add1(tacc + a, tloc[a]);
    }
    if (tb)
        for (int a = 0; a < 3; ++a) tb[a] += tacc[a];
}

/* CS_VorticityConfinement.glsl:133-167 reversed: velb of the final velocity
 * -> posb (accumulated, committed positions) and omb (adjoint of omega). */
static void vorticity_vjp(const orc_params* p, uint32_t n, const orc_real* pos, const orc_real* om,
                          const uint32_t* ids, const int32_t* table, const orc_real* velb, orc_real* posb, orc_real* omb)
{
    orc_real* magb = (orc_real*)calloc((size_t)n, sizeof(orc_real));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const orc_real* xi = pos + 3 * i;
        orc_real eta[3] = {0, 0, 0};
        ADJ_FOR_EACH(p, xi, i, ids, table, {
            const orc_real* xj = pos + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            if (r2 <= p->h2 && r2 >= 1e-10) {
                const orc_real k = sqrt(dot3(om + 3 * j, om + 3 * j)) * spiky_s(p, r2);
                for (int a = 0; a < 3; ++a) eta[a] += r[a] * k;
            }
        });
        for (int a = 0; a < 3; ++a) eta[a] *= p->inv_rho0;
        const orc_real el = sqrt(dot3(eta, eta));
        if (el < 1e-6) continue;
        const orc_real N[3] = {eta[0] / el, eta[1] / el, eta[2] / el};
        const orc_real* w = om + 3 * i;
        const orc_real k = p->vort_eps * p->dt;
        const orc_real yb[3] = {k * velb[3 * i], k * velb[3 * i + 1], k * velb[3 * i + 2]};
        /* y = N x w */
        const orc_real Nb[3] = {w[1] * yb[2] - w[2] * yb[1], w[2] * yb[0] - w[0] * yb[2], w[0] * yb[1] - w[1] * yb[0]};
        const orc_real wb[3] = {yb[1] * N[2] - yb[2] * N[1], yb[2] * N[0] - yb[0] * N[2], yb[0] * N[1] - yb[1] * N[0]};
        for (int a = 0; a < 3; ++a) atomic_add1(omb + 3 * i + a, wb[a]);
        const orc_real nn = dot3(N, Nb);
        orc_real eb[3];
        for (int a = 0; a < 3; ++a) eb[a] = (Nb[a] - N[a] * nn) / el * p->inv_rho0;
        orc_real own[3] = {0, 0, 0};
        ADJ_FOR_EACH(p, xi, i, ids, table, {
            const orc_real* xj = pos + 3 * j;
            const orc_real r[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
            const orc_real r2 = dot3(r, r);
            if (r2 <= p->h2 && r2 >= 1e-10) {
                const orc_real mag = sqrt(dot3(om + 3 * j, om + 3 * j));
                const orc_real s_ = spiky_s(p, r2);
                atomic_add1(magb + j, s_ * dot3(r, eb));
                orc_real rb[3] = {0, 0, 0};
                const orc_real gb[3] = {mag * eb[0], mag * eb[1], mag * eb[2]};
                grad_vjp(p, r, r2, gb, rb);
                for (int a = 0; a < 3; ++a) own[a] += rb[a];
                atomic_sub3(posb + 3 * j, rb);
            }
        });
        for (int a = 0; a < 3; ++a) atomic_add1(posb + 3 * i + a, own[a]);
    }
    for (uint32_t j = 0; j < n; ++j) {
        const orc_real mag = sqrt(dot3(om + 3 * j, om + 3 * j));
        if (mag > 0.0)
            for (int a = 0; a < 3; ++a) omb[3 * j + a] += magb[j] * om[3 * j + a] / mag;
    }
    free(magb);
}

/* ---- one step: forward with checkpoints, then reverse ---------------------- */
typedef struct {
    orc_real *xs, *lam; /* (I+1) x n x 3 positions, I x n lambdas */
    orc_real *vp, *x0;
    uint32_t *keys, *sk, *ids;
    int32_t* table;
} subrec;

/* Recompute one substep from (pos, vel) at its start, recording what the
 * reverse needs; pos/vel are advanced to the substep end (omega filled). */
static void substep_record(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* pos, orc_real* vel,
                           orc_real* omega, subrec* R)
{
    const uint32_t I = p->iterations;
    memcpy(R->x0, pos, sizeof(orc_real) * 3 * n);
    orc_predict(p, n, pos, vel, R->xs, R->keys);
    memcpy(R->vp, vel, sizeof(orc_real) * 3 * n);
    orc_stable_sort(R->keys, n, p->hash_size, R->sk, R->ids);
    orc_build_table(R->sk, n, p->hash_size, R->table);
    for (uint32_t it = 1; it <= I; ++it) {
        orc_real* xprev = R->xs + (size_t)(it - 1) * 3 * n;
        orc_real* xnext = R->xs + (size_t)it * 3 * n;
        orc_real* lam = R->lam + (size_t)(it - 1) * n;
        orc_lambda(p, n, xprev, R->ids, R->table, NULL, it, lam, NULL);
        memcpy(xnext, xprev, sizeof(orc_real) * 3 * n);
        orc_deltap_apply(p, s, n, xnext, lam, R->ids, R->table, NULL, it, NULL);
    }
    orc_integrate(p, s, n, pos, vel, R->xs + (size_t)I * 3 * n, R->ids, R->table, omega);
}

void orc_adjoint_step(const orc_params* p, const orc_sdf* s, uint32_t n, const orc_real* pos0, const orc_real* vel0,
                      const orc_real* gpos, const orc_real* gvel, orc_real* gpos0, orc_real* gvel0, orc_real* gt,
                      orc_real* pos_out, orc_real* vel_out)
{
    const uint32_t S = p->substeps, I = p->iterations;
    const size_t n3 = 3 * (size_t)n;
    orc_real* cp_pos = (orc_real*)malloc(sizeof(orc_real) * n3 * S);
    orc_real* cp_vel = (orc_real*)malloc(sizeof(orc_real) * n3 * S);
    orc_real* pos = (orc_real*)malloc(sizeof(orc_real) * n3);
    orc_real* vel = (orc_real*)malloc(sizeof(orc_real) * n3);
    orc_real* om = (orc_real*)calloc(n3, sizeof(orc_real));
    subrec R;
    R.xs = (orc_real*)malloc(sizeof(orc_real) * n3 * (I + 1));
    R.lam = (orc_real*)malloc(sizeof(orc_real) * (size_t)n * (I ? I : 1));
    R.vp = (orc_real*)malloc(sizeof(orc_real) * n3);
    R.x0 = (orc_real*)malloc(sizeof(orc_real) * n3);
    R.keys = (uint32_t*)malloc(sizeof(uint32_t) * n);
    R.sk = (uint32_t*)malloc(sizeof(uint32_t) * n);
    R.ids = (uint32_t*)malloc(sizeof(uint32_t) * n);
    R.table = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)p->hash_size);
    if (gt) gt[0] = gt[1] = gt[2] = 0.0;

    /* forward with per-substep checkpoints */
    memcpy(pos, pos0, sizeof(orc_real) * n3);
    memcpy(vel, vel0, sizeof(orc_real) * n3);
    for (uint32_t sub = 0; sub < S; ++sub) {
        memcpy(cp_pos + sub * n3, pos, sizeof(orc_real) * n3);
        memcpy(cp_vel + sub * n3, vel, sizeof(orc_real) * n3);
        substep_record(p, s, n, pos, vel, om, &R);
    }
    if (p->vort_on) orc_vorticity(p, n, pos, vel, om, R.ids, R.table);
    if (pos_out) memcpy(pos_out, pos, sizeof(orc_real) * n3);
    if (vel_out) memcpy(vel_out, vel, sizeof(orc_real) * n3);

    /* reverse */
    orc_real* pb = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* vb = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* omb = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* xsb = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* xsb2 = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* vpb = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* x0b = (orc_real*)calloc(n3, sizeof(orc_real));
    orc_real* lamb = (orc_real*)calloc((size_t)n, sizeof(orc_real));
    if (gpos) memcpy(pb, gpos, sizeof(orc_real) * n3);
    if (gvel) memcpy(vb, gvel, sizeof(orc_real) * n3);
    for (int sub = (int)S - 1; sub >= 0; --sub) {
        memcpy(pos, cp_pos + sub * n3, sizeof(orc_real) * n3);
        memcpy(vel, cp_vel + sub * n3, sizeof(orc_real) * n3);
        substep_record(p, s, n, pos, vel, om, &R);
        memset(omb, 0, sizeof(orc_real) * n3);
        if (sub == (int)S - 1 && p->vort_on) vorticity_vjp(p, n, pos, om, R.ids, R.table, vb, pb, omb);
        memset(xsb, 0, sizeof(orc_real) * n3);
        memset(vpb, 0, sizeof(orc_real) * n3);
        memset(x0b, 0, sizeof(orc_real) * n3);
        integrate_vjp(p, s, n, R.xs + (size_t)I * n3, R.vp, R.x0, R.ids, R.table, pb, vb,
                      p->vort_on ? omb : NULL, xsb, vpb, x0b, gt);
        for (int it = (int)I; it >= 1; --it) {
            const orc_real* xprev = R.xs + (size_t)(it - 1) * n3;
            const orc_real* lam = R.lam + (size_t)(it - 1) * n;
            memset(xsb2, 0, sizeof(orc_real) * n3);
            memset(lamb, 0, sizeof(orc_real) * n);
            deltap_vjp(p, s, n, xprev, lam, R.ids, R.table, xsb, xsb2, lamb, gt);
            lambda_vjp(p, n, xprev, R.ids, R.table, lamb, xsb2);
            orc_real* t = xsb;
            xsb = xsb2;
            xsb2 = t;
        }
        /* CS_PredictAndHash.glsl:102,114 reversed */
        for (size_t k = 0; k < n3; ++k) {
            vb[k] = vpb[k] + p->dt * xsb[k];
            pb[k] = xsb[k] + x0b[k];
        }
    }
    if (gpos0) memcpy(gpos0, pb, sizeof(orc_real) * n3);
    if (gvel0) memcpy(gvel0, vb, sizeof(orc_real) * n3);
    free(pb); free(vb); free(omb); free(xsb); free(xsb2); free(vpb); free(x0b); free(lamb);
    free(cp_pos); free(cp_vel); free(pos); free(vel); free(om);
    free(R.xs); free(R.lam); free(R.vp); free(R.x0); free(R.keys); free(R.sk); free(R.ids); free(R.table);
}
