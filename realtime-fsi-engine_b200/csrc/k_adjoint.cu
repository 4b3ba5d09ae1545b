// k_adjoint.cu — reverse-mode kernels of the PBF substep (multi-scene engine).
//
// The backward of one substep runs on the state the forward recorded for it
// (recomputed from the substep's checkpoint): sorted slots, the cell table,
// every iteration's (x*, lambda) with the lambda denominators and raw dp.
// Each kernel is one thread per particle in the forward's processing order;
// it recomputes what it needs of its own particle, accumulates its own
// adjoint in registers and scatters the neighbour's share of every pair term
// with atomic adds (sm_90+ float4 atomics), walking the same 27 buckets with
// the same multiplicity and order as the forward.  Discrete choices (neighbour
// sets, wall/SDF contacts, clamps) are the forward's, replayed.
//
// Derivatives (r = x_i - x_j, q = |r|, W = poly6, grad W = r s(r^2)):
//   dW/d(r^2)  = -3 K6 (h^2 - r^2)^2
//   ds/d(r^2)  = Ks (h - q)(h + q) / (2 q^3)          (s = -Ks (h - q)^2 / q)
//   adjoint of a = r s given a_bar: r_bar = s a_bar + 2 ds (r . a_bar) r
#include "masked_body.cuh"
#include "pbf_batch.h"

namespace pbf {

constexpr int kAThreads = 128;
// The reverse pair passes and the recording Δp are held to 8 resident blocks
// (at most 64 registers).  Left to itself the compiler gave the Δp adjoint 56
// registers and 1.2 KB of spills; at 8 blocks the backward of one step (16
// substeps x 4 iterations) of 16 scenes of 32,768 particles takes 42.4 ms
// instead of 46.0 (10 or 12 blocks: 44.1 / 45.2 ms; 4: 49.5).
constexpr int kAdjBlocks = 8;

__device__ __forceinline__ float poly6_d(const DevParams& P, float r2)
{
    const float d = P.h2 - r2;
    return -3.0f * P.poly6 * d * d;
}

__device__ __forceinline__ float spiky_ds(const DevParams& P, float r2)
{
    const float inv = rsqrtf(r2);
    const float q = r2 * inv;
    return P.spiky * (P.h - q) * (P.h + q) * 0.5f * inv * inv * inv;
}

// d s_corr / d(r^2) (CS_ComputeDeltaP.glsl:94-104), r2 < h2
__device__ __forceinline__ float scorr_d(const DevParams& P, float r2)
{
    const float d = P.h2 - r2;
    const float w = P.poly6 * d * d * d;
    if (!(P.wq > 1e-12f && w > 0.0f)) return 0.0f;
    const float ratio = w * P.inv_wq;
    float pw;
    if (P.ncorr_is4) {
        pw = ratio * ratio * ratio * 4.0f;
    } else {
        pw = P.n_corr * powf(ratio, P.n_corr - 1.0f);
    }
    return -P.k_corr * pw * P.inv_wq * poly6_d(P, r2);
}

__device__ __forceinline__ float3 grad_vjp(const DevParams& P, float rx, float ry, float rz, float r2, float3 ab)
{
    const float s = spiky_scale(P, r2);
    const float k = 2.0f * spiky_ds(P, r2) * (rx * ab.x + ry * ab.y + rz * ab.z);
    return make_float3(s * ab.x + k * rx, s * ab.y + k * ry, s * ab.z + k * rz);
}

__device__ __forceinline__ void add_own(float4* p, float3 v, float w)
{
    atomicAdd(p, make_float4(v.x, v.y, v.z, w));
}

// ---- SDF: analytic gradient of the clamped trilinear interpolant -------------------------
__device__ __forceinline__ float3 sdf_grad_exact(const SdfDev& S, float px, float py, float pz)
{
    const float u = (px - S.ox) * S.inv_cell, v = (py - S.oy) * S.inv_cell, w = (pz - S.oz) * S.inv_cell;
    const float hx = (float)(S.dx - 1), hy = (float)(S.dy - 1), hz = (float)(S.dz - 1);
    const bool lx = u > 0.0f && u < hx, ly = v > 0.0f && v < hy, lz = w > 0.0f && w < hz;
    const float uc = fminf(fmaxf(u, 0.0f), hx), vc = fminf(fmaxf(v, 0.0f), hy), wc = fminf(fmaxf(w, 0.0f), hz);
    const float fu = floorf(uc), fv = floorf(vc), fw = floorf(wc);
    const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
    const int i1 = min(i0 + 1, S.dx - 1), j1 = min(j0 + 1, S.dy - 1), k1 = min(k0 + 1, S.dz - 1);
    const float a = uc - fu, b = vc - fv, c = wc - fw;
    const float c000 = sdf_texel(S, i0, j0, k0), c001 = sdf_texel(S, i0, j0, k1);
    const float c010 = sdf_texel(S, i0, j1, k0), c011 = sdf_texel(S, i0, j1, k1);
    const float c100 = sdf_texel(S, i1, j0, k0), c101 = sdf_texel(S, i1, j0, k1);
    const float c110 = sdf_texel(S, i1, j1, k0), c111 = sdf_texel(S, i1, j1, k1);
    const float c00 = c000 + (c001 - c000) * c, c01 = c010 + (c011 - c010) * c;
    const float c10 = c100 + (c101 - c100) * c, c11 = c110 + (c111 - c110) * c;
    const float c0 = c00 + (c01 - c00) * b, c1 = c10 + (c11 - c10) * b;
    const float da = c1 - c0;
    const float db = (1.0f - a) * (c01 - c00) + a * (c11 - c10);
    const float dc = (1.0f - a) * ((1.0f - b) * (c001 - c000) + b * (c011 - c010)) +
                     a * ((1.0f - b) * (c101 - c100) + b * (c111 - c110));
    return make_float3(lx ? da * S.inv_cell : 0.0f, ly ? db * S.inv_cell : 0.0f, lz ? dc * S.inv_cell : 0.0f);
}

// Vector-Jacobian product of sdf_project at input x: xb (adjoint of the
// projected point) becomes the adjoint of x, nb is the adjoint of the push
// normal; the translation adjoint (minus the SDF-dependent part) is
// returned through tb.  Branches are taken exactly as sdf_project takes them.
__device__ __forceinline__ bool project_vjp(const SdfDev& S, float3 x, float3& xb, float3 nb, float3& tb)
{
    if (sdf_far_obstacle(S, x.x, x.y, x.z)) return false;
    const float e = S.cell;
    const float d = sdf_sample(S, x.x, x.y, x.z);
    if (S.containment ? !(d > -S.padding) : !(d < S.padding)) return false;  // no contact
    const float inv2e = 1.0f / (2.0f * e);
    const float gx = (sdf_sample(S, x.x + e, x.y, x.z) - sdf_sample(S, x.x - e, x.y, x.z)) * inv2e;
    const float gy = (sdf_sample(S, x.x, x.y + e, x.z) - sdf_sample(S, x.x, x.y - e, x.z)) * inv2e;
    const float gz = (sdf_sample(S, x.x, x.y, x.z + e) - sdf_sample(S, x.x, x.y, x.z - e)) * inv2e;
    const float len = sqrtf(gx * gx + gy * gy + gz * gz);
    if (!(len > 1e-6f)) return false;
    float sgn, sc;
    if (S.containment) {
        if (!(d > -S.padding)) return false;
        sgn = -1.0f;
        sc = d + S.padding;
    } else {
        if (!(d < S.padding)) return false;
        sgn = 1.0f;
        sc = S.padding - d;
    }
    const float3 n = make_float3(sgn * gx / len, sgn * gy / len, sgn * gz / len);
    // rows of H = dG/dx from the analytic gradients of the six samples
    const float3 hxp = sdf_grad_exact(S, x.x + e, x.y, x.z), hxm = sdf_grad_exact(S, x.x - e, x.y, x.z);
    const float3 hyp = sdf_grad_exact(S, x.x, x.y + e, x.z), hym = sdf_grad_exact(S, x.x, x.y - e, x.z);
    const float3 hzp = sdf_grad_exact(S, x.x, x.y, x.z + e), hzm = sdf_grad_exact(S, x.x, x.y, x.z - e);
    const float3 H0 = make_float3((hxp.x - hxm.x) * inv2e, (hxp.y - hxm.y) * inv2e, (hxp.z - hxm.z) * inv2e);
    const float3 H1 = make_float3((hyp.x - hym.x) * inv2e, (hyp.y - hym.y) * inv2e, (hyp.z - hym.z) * inv2e);
    const float3 H2 = make_float3((hzp.x - hzm.x) * inv2e, (hzp.y - hzm.y) * inv2e, (hzp.z - hzm.z) * inv2e);
    const float3 gq = sdf_grad_exact(S, x.x, x.y, x.z);
    const float3 v = make_float3(sc * xb.x + nb.x, sc * xb.y + nb.y, sc * xb.z + nb.z);
    const float nv = n.x * v.x + n.y * v.y + n.z * v.z;
    const float k = sgn / len;
    const float3 pv = make_float3((v.x - n.x * nv) * k, (v.y - n.y * nv) * k, (v.z - n.z * nv) * k);
    const float nxb = n.x * xb.x + n.y * xb.y + n.z * xb.z;
    const float gs = S.containment ? nxb : -nxb;
    const float3 add = make_float3(H0.x * pv.x + H1.x * pv.y + H2.x * pv.z + gq.x * gs,
                                   H0.y * pv.x + H1.y * pv.y + H2.y * pv.z + gq.y * gs,
                                   H0.z * pv.x + H1.z * pv.y + H2.z * pv.z + gq.z * gs);
    xb = make_float3(xb.x + add.x, xb.y + add.y, xb.z + add.z);
    tb = make_float3(tb.x - add.x, tb.y - add.y, tb.z - add.z);
    return true;
}

__device__ __forceinline__ void add_t(float* tgrad, int k, float3 tb)
{
    if (tb.x != 0.0f) atomicAdd(tgrad + 4 * k + 0, tb.x);
    if (tb.y != 0.0f) atomicAdd(tgrad + 4 * k + 1, tb.y);
    if (tb.z != 0.0f) atomicAdd(tgrad + 4 * k + 2, tb.z);
}

#define AD_PROLOGUE                                                                                 \
    const int t = blockIdx.x * blockDim.x + threadIdx.x;                                            \
    if (t >= (int)P.n) return;                                                                      \
    const int s = order ? (int)__ldg(order + t) : t;                                                \
    const int sid = (int)__ldg(scene_of + t);                                                       \
    const SceneDev* SC = scenes + sid;                                                              \
    const int2* tab = table + __ldg(&SC->table_off);                                                \
    const uint32_t mask = __ldg(&SC->mask);

// ---- recording forward passes -------------------------------------------------------------
__global__ void __launch_bounds__(kAThreads) k_ad_lambda_rec(DevParams P, const SceneDev* __restrict__ scenes,
                                                             const uint16_t* __restrict__ scene_of,
                                                             const uint32_t* __restrict__ order,
                                                             const int2* __restrict__ table,
                                                             const float4* __restrict__ xin, float4* __restrict__ xl,
                                                             float4* __restrict__ auxl, float* __restrict__ rhol)
{
    AD_PROLOGUE
    float rho, den;
    float3 g;
    xl[s] = lambda_particle_x(P, tab, mask, xin, s, rho, g, den);
    auxl[s] = make_float4(g.x, g.y, g.z, den);
    rhol[s] = rho;
}

__global__ void __launch_bounds__(kAThreads, kAdjBlocks) k_ad_deltap_rec(DevParams P, const SceneDev* __restrict__ scenes,
                                                             const uint16_t* __restrict__ scene_of,
                                                             const uint32_t* __restrict__ order,
                                                             const int2* __restrict__ table,
                                                             const float4* __restrict__ xl, float4* __restrict__ xout,
                                                             float4* __restrict__ auxd)
{
    AD_PROLOGUE
    const SdfDev sdf = load_sdf(SC);
    float3 dp;
    xout[s] = deltap_particle_x(P, tab, mask, sdf, xl, s, dp);
    auxd[s] = make_float4(dp.x, dp.y, dp.z, 0.0f);
}

// ---- CS_VorticityConfinement.glsl:133-167 reversed -----------------------------------------
// velb (particle order) -> posb_s (sorted, committed positions) and omb
// (sorted: xyz adjoint of omega_i, w adjoint of |omega_j| by scatter).
__global__ void __launch_bounds__(kAThreads) k_ad_vorticity(DevParams P, const SceneDev* __restrict__ scenes,
                                                            const uint16_t* __restrict__ scene_of,
                                                            const uint32_t* __restrict__ order,
                                                            const int2* __restrict__ table,
                                                            const float4* __restrict__ spos,
                                                            const float4* __restrict__ somega,
                                                            const uint32_t* __restrict__ ids,
                                                            const float4* __restrict__ velb,
                                                            float4* __restrict__ posb_s, float4* __restrict__ omb)
{
    AD_PROLOGUE
    const float4 xi = __ldg(spos + s);
    float ex = 0.f, ey = 0.f, ez = 0.f;
    auto hit = [&](float r2) { return r2 <= P.h2 && r2 >= 1e-10f; };
    masked_walk(P, tab, mask, spos, xi.x, xi.y, xi.z, s, hit, [&](int k) {
        const float4 xj = __ldg(spos + k);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        const float sc = spiky_scale(P, r2) * __ldg(&somega[k].w);
        ex += rx * sc;
        ey += ry * sc;
        ez += rz * sc;
    });
    ex *= P.inv_rho0;
    ey *= P.inv_rho0;
    ez *= P.inv_rho0;
    const float el = sqrtf(ex * ex + ey * ey + ez * ez);
    if (el < 1e-6f) return;
    const float3 N = make_float3(ex / el, ey / el, ez / el);
    const float4 w = __ldg(somega + s);
    const float4 vb4 = __ldg(velb + __ldg(ids + s));
    const float k = P.vort_eps * P.dt;
    const float3 yb = make_float3(k * vb4.x, k * vb4.y, k * vb4.z);
    // y = N x w:  N_bar = w x y_bar,  w_bar = y_bar x N
    const float3 Nb = make_float3(w.y * yb.z - w.z * yb.y, w.z * yb.x - w.x * yb.z, w.x * yb.y - w.y * yb.x);
    const float3 wb = make_float3(yb.y * N.z - yb.z * N.y, yb.z * N.x - yb.x * N.z, yb.x * N.y - yb.y * N.x);
    add_own(omb + s, wb, 0.0f);
    const float nn = N.x * Nb.x + N.y * Nb.y + N.z * Nb.z;
    const float ke = P.inv_rho0 / el;
    const float3 eb = make_float3((Nb.x - N.x * nn) * ke, (Nb.y - N.y * nn) * ke, (Nb.z - N.z * nn) * ke);
    float3 own = make_float3(0.f, 0.f, 0.f);
    masked_walk(P, tab, mask, spos, xi.x, xi.y, xi.z, s, hit, [&](int k2) {
        const float4 xj = __ldg(spos + k2);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        const float mag = __ldg(&somega[k2].w);
        const float sg = spiky_scale(P, r2);
        const float3 rb = grad_vjp(P, rx, ry, rz, r2, make_float3(mag * eb.x, mag * eb.y, mag * eb.z));
        own.x += rb.x;
        own.y += rb.y;
        own.z += rb.z;
        atomicAdd(posb_s + k2, make_float4(-rb.x, -rb.y, -rb.z, 0.0f));
        atomicAdd(&omb[k2].w, sg * (rx * eb.x + ry * eb.y + rz * eb.z));
    });
    add_own(posb_s + s, own, 0.0f);
}

// ---- CS_Integrate.glsl:135-280 reversed -------------------------------------------------------
// (posb, velb) particle order (+ posb_s sorted, omb sorted when the vorticity
// pass was reversed) -> gx (adjoint of x*), gv (of v'), x0b, tgrad.
__global__ void __launch_bounds__(kAThreads, kAdjBlocks) k_ad_integrate(
    DevParams P, const SceneDev* __restrict__ scenes, const uint16_t* __restrict__ scene_of,
    const uint32_t* __restrict__ order, const int2* __restrict__ table, const float4* __restrict__ xs,
    const float4* __restrict__ sv, const float4* __restrict__ cp_pos, const uint32_t* __restrict__ ids,
    const float4* __restrict__ posb, const float4* __restrict__ velb, const float4* __restrict__ posb_s,
    const float4* __restrict__ omb, const float4* __restrict__ somega, float4* __restrict__ gx,
    float4* __restrict__ gv, float4* __restrict__ x0b, float* __restrict__ tgrad)
{
    AD_PROLOGUE
    const SdfDev sdf = load_sdf(SC);
    const float4 x4 = __ldg(xs + s);
    const float4 v0 = __ldg(sv + s);
    const uint32_t id = __ldg(ids + s);
    const float4 p0 = __ldg(cp_pos + id);
    float fx = 0.f, fy = 0.f, fz = 0.f;
    if (P.visc_on) {
        masked_walk(P, tab, mask, xs, x4.x, x4.y, x4.z, s, [&](float r2) { return r2 <= P.h2; }, [&](int k) {
            const float4 xj = __ldg(xs + k);
            const float rx = x4.x - xj.x, ry = x4.y - xj.y, rz = x4.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            const float4 vj = __ldg(sv + k);
            const float w = poly6_in(P, r2) * P.inv_rho0;
            fx += (vj.x - v0.x) * w;
            fy += (vj.y - v0.y) * w;
            fz += (vj.z - v0.z) * w;
        });
    }
    float bmin[3], bmax[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        bmin[a] = __ldg(&SC->bmin[a]);
        bmax[a] = __ldg(&SC->bmax[a]);
    }
    float3 x = make_float3(x4.x, x4.y, x4.z);
    bool colx = false, coly = false, colz = false;
    if (x.x <= bmin[0]) { x.x = bmin[0]; colx = true; }
    if (x.x >= bmax[0]) { x.x = bmax[0]; colx = true; }
    if (x.y <= bmin[1]) { x.y = bmin[1]; coly = true; }
    if (x.y >= bmax[1]) { x.y = bmax[1]; coly = true; }
    if (x.z <= bmin[2]) { x.z = bmin[2]; colz = true; }
    if (x.z >= bmax[2]) { x.z = bmax[2]; colz = true; }
    const float3 xw = x;
    bool col_sdf = false;
    float3 nrm = make_float3(0.f, 0.f, 0.f);
    if (sdf.enabled) col_sdf = sdf_project(sdf, x, nrm);
    float vdx = 0.f, vdy = 0.f, vdz = 0.f;
    if (P.visc_on) {
        vdx = fx * P.viscosity;
        vdy = fy * P.viscosity;
        vdz = fz * P.viscosity;
    }
    const float v1x = (x.x - p0.x) * P.inv_dt + vdx, v1y = (x.y - p0.y) * P.inv_dt + vdy,
                v1z = (x.z - p0.z) * P.inv_dt + vdz;
    const float sp2 = v1x * v1x + v1y * v1y + v1z * v1z;
    float v2x = v1x, v2y = v1y, v2z = v1z;
    if (sp2 > 2500.0f) {
        const float sc = 50.0f / sqrtf(sp2);
        v2x *= sc;
        v2y *= sc;
        v2z *= sc;
    }
    const float v3x = colx ? v2x * -P.damping : v2x, v3y = coly ? v2y * -P.damping : v2y,
                v3z = colz ? v2z * -P.damping : v2z;
    // reverse
    const float4 vb4 = __ldg(velb + id);
    float3 vb = make_float3(vb4.x, vb4.y, vb4.z);
    float3 nb = make_float3(0.f, 0.f, 0.f);
    if (col_sdf) {
        const float vn = v3x * nrm.x + v3y * nrm.y + v3z * nrm.z;
        const float nvb = nrm.x * vb.x + nrm.y * vb.y + nrm.z * vb.z;
        nb = make_float3(-(vn * vb.x + nvb * v3x), -(vn * vb.y + nvb * v3y), -(vn * vb.z + nvb * v3z));
        vb = make_float3(vb.x - nrm.x * nvb, vb.y - nrm.y * nvb, vb.z - nrm.z * nvb);
    }
    if (colx) vb.x *= -P.damping;
    if (coly) vb.y *= -P.damping;
    if (colz) vb.z *= -P.damping;
    if (sp2 > 2500.0f) {
        const float len = sqrtf(sp2);
        const float ux = v1x / len, uy = v1y / len, uz = v1z / len;
        const float ub = ux * vb.x + uy * vb.y + uz * vb.z;
        const float k = 50.0f / len;
        vb = make_float3(k * (vb.x - ux * ub), k * (vb.y - uy * ub), k * (vb.z - uz * ub));
    }
    const float4 pb4 = __ldg(posb + id);
    float3 xb = make_float3(pb4.x + vb.x * P.inv_dt, pb4.y + vb.y * P.inv_dt, pb4.z + vb.z * P.inv_dt);
    if (posb_s) {
        const float4 q = posb_s[s];
        xb.x += q.x;
        xb.y += q.y;
        xb.z += q.z;
    }
    x0b[s] = make_float4(-vb.x * P.inv_dt, -vb.y * P.inv_dt, -vb.z * P.inv_dt, 0.0f);
    float3 tb = make_float3(0.f, 0.f, 0.f);
    if (col_sdf) project_vjp(sdf, xw, xb, nb, tb);
    add_t(tgrad, sid, tb);
    float3 own = make_float3(colx ? 0.f : xb.x, coly ? 0.f : xb.y, colz ? 0.f : xb.z);
    float3 vfb = make_float3(0.f, 0.f, 0.f), cb = make_float3(0.f, 0.f, 0.f);
    if (P.visc_on) vfb = make_float3(vb.x * P.viscosity, vb.y * P.viscosity, vb.z * P.viscosity);
    if (P.vort_on && omb) {
        const float4 o = omb[s];
        const float4 w = __ldg(somega + s);
        float kx = 0.f;
        if (w.w > 0.0f) kx = o.w / w.w;
        cb = make_float3((o.x + kx * w.x) * P.inv_rho0, (o.y + kx * w.y) * P.inv_rho0, (o.z + kx * w.z) * P.inv_rho0);
    }
    float3 vown = make_float3(0.f, 0.f, 0.f);
    const bool need_walk = P.visc_on || (P.vort_on && omb);
    if (need_walk) {
        masked_walk(P, tab, mask, xs, x4.x, x4.y, x4.z, s, [&](float r2) { return r2 <= P.h2; }, [&](int k) {
            const float4 xj = __ldg(xs + k);
            const float rx = x4.x - xj.x, ry = x4.y - xj.y, rz = x4.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            const float4 vj = __ldg(sv + k);
            const float ux = vj.x - v0.x, uy = vj.y - v0.y, uz = vj.z - v0.z;
            float3 ub = make_float3(0.f, 0.f, 0.f), rb = make_float3(0.f, 0.f, 0.f);
            if (P.visc_on) {
                const float w = poly6_in(P, r2) * P.inv_rho0;
                ub = make_float3(vfb.x * w, vfb.y * w, vfb.z * w);
                const float kk = (vfb.x * ux + vfb.y * uy + vfb.z * uz) * P.inv_rho0 * poly6_d(P, r2) * 2.0f;
                rb = make_float3(kk * rx, kk * ry, kk * rz);
            }
            if (P.vort_on && omb && r2 >= 1e-10f) {
                const float sg = spiky_scale(P, r2);
                const float gx_ = rx * sg, gy_ = ry * sg, gz_ = rz * sg;
                ub.x += gy_ * cb.z - gz_ * cb.y;
                ub.y += gz_ * cb.x - gx_ * cb.z;
                ub.z += gx_ * cb.y - gy_ * cb.x;
                const float3 gb = make_float3(cb.y * uz - cb.z * uy, cb.z * ux - cb.x * uz, cb.x * uy - cb.y * ux);
                const float3 r2b = grad_vjp(P, rx, ry, rz, r2, gb);
                rb.x += r2b.x;
                rb.y += r2b.y;
                rb.z += r2b.z;
            }
            own.x += rb.x;
            own.y += rb.y;
            own.z += rb.z;
            vown.x -= ub.x;
            vown.y -= ub.y;
            vown.z -= ub.z;
            atomicAdd(gx + k, make_float4(-rb.x, -rb.y, -rb.z, 0.0f));
            atomicAdd(gv + k, make_float4(ub.x, ub.y, ub.z, 0.0f));
        });
    }
    add_own(gx + s, own, 0.0f);
    add_own(gv + s, vown, 0.0f);
}

// ---- CS_ComputeDeltaP.glsl:120-166 + CS_ApplyDeltaP.glsl:80-124 reversed --------------------
// gin (adjoint of this iteration's output x*) -> gout.xyz (adjoint of the
// input x*) and gout.w (adjoint of lambda), tgrad.
__global__ void __launch_bounds__(kAThreads, kAdjBlocks) k_ad_deltap(DevParams P, const SceneDev* __restrict__ scenes,
                                                         const uint16_t* __restrict__ scene_of,
                                                         const uint32_t* __restrict__ order,
                                                         const int2* __restrict__ table,
                                                         const float4* __restrict__ xl,
                                                         const float4* __restrict__ auxd,
                                                         const float4* __restrict__ gin, float4* __restrict__ gout,
                                                         float* __restrict__ tgrad)
{
    AD_PROLOGUE
    const float4 xi = __ldg(xl + s);
    const float4 g4 = gin[s];
    const float4 dp = __ldg(auxd + s);
    float dx = dp.x, dy = dp.y, dz = dp.z;
    const float l2 = dx * dx + dy * dy + dz * dz;
    const bool clamped = l2 > P.max_dp * P.max_dp;
    if (clamped) {
        const float sc = P.max_dp * rsqrtf(l2);
        dx *= sc;
        dy *= sc;
        dz *= sc;
    }
    const float3 x = make_float3(xi.x + dx, xi.y + dy, xi.z + dz);
    float3 xb = make_float3(g4.x, g4.y, g4.z);
    const SdfDev sdf = load_sdf(SC);
    if (sdf.enabled) {
        float3 tb = make_float3(0.f, 0.f, 0.f);
        project_vjp(sdf, x, xb, make_float3(0.f, 0.f, 0.f), tb);
        add_t(tgrad, sid, tb);
    }
    float3 dpb = xb;
    if (clamped) {
        const float len = sqrtf(l2);
        const float ux = dp.x / len, uy = dp.y / len, uz = dp.z / len;
        const float ub = ux * xb.x + uy * xb.y + uz * xb.z;
        const float k = P.max_dp / len;
        dpb = make_float3(k * (xb.x - ux * ub), k * (xb.y - uy * ub), k * (xb.z - uz * ub));
    }
    const float3 accb = make_float3(dpb.x * P.inv_rho0, dpb.y * P.inv_rho0, dpb.z * P.inv_rho0);
    float3 own = xb;
    float lown = 0.0f;
    const float li = xi.w;
    masked_walk(P, tab, mask, xl, xi.x, xi.y, xi.z, s, [&](float r2) { return r2 <= P.h2 && r2 >= 1e-10f; },
                [&](int k) {
                    const float4 xj = __ldg(xl + k);
                    const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                    const float r2 = rx * rx + ry * ry + rz * rz;
                    const float sg = spiky_scale(P, r2);
                    float f = li + xj.w;
                    if (P.scorr) f += scorr_term(P, r2);
                    const float ga = sg * (rx * accb.x + ry * accb.y + rz * accb.z);
                    lown += ga;
                    float3 rb = grad_vjp(P, rx, ry, rz, r2, make_float3(f * accb.x, f * accb.y, f * accb.z));
                    if (P.scorr) {
                        const float kk = ga * scorr_d(P, r2) * 2.0f;
                        rb.x += kk * rx;
                        rb.y += kk * ry;
                        rb.z += kk * rz;
                    }
                    own.x += rb.x;
                    own.y += rb.y;
                    own.z += rb.z;
                    atomicAdd(gout + k, make_float4(-rb.x, -rb.y, -rb.z, ga));
                });
    add_own(gout + s, own, lown);
}

// ---- CS_ComputeLambdas.glsl:108-162 reversed: gout.w (lambda adjoint) -> gout.xyz ---------------
__global__ void __launch_bounds__(kAThreads, kAdjBlocks) k_ad_lambda(DevParams P, const SceneDev* __restrict__ scenes,
                                                         const uint16_t* __restrict__ scene_of,
                                                         const uint32_t* __restrict__ order,
                                                         const int2* __restrict__ table,
                                                         const float4* __restrict__ xl,
                                                         const float4* __restrict__ auxl,
                                                         const float* __restrict__ rhol, float4* __restrict__ gout)
{
    AD_PROLOGUE
    const float lb = gout[s].w;
    if (lb == 0.0f) return;
    const float4 xi = __ldg(xl + s);
    const float4 aux = __ldg(auxl + s);
    const float rho = __ldg(rhol + s);
    const float craw = rho / P.rho0 - 1.0f;
    const float C = fmaxf(craw, -P.cohesion);
    const float den = aux.w;
    const float Cb = -lb / den;
    const float Db = lb * C / (den * den);
    const float rhob = (craw < -P.cohesion) ? 0.0f : Cb / P.rho0;
    const float3 gsb = make_float3(Db * 2.0f * aux.x * P.inv_rho0, Db * 2.0f * aux.y * P.inv_rho0,
                                   Db * 2.0f * aux.z * P.inv_rho0);
    const float k2 = Db * 2.0f * P.inv_rho0_sq;
    float3 own = make_float3(0.f, 0.f, 0.f);
    masked_walk(P, tab, mask, xl, xi.x, xi.y, xi.z, s, [&](float r2) { return r2 <= P.h2; }, [&](int k) {
        const float4 xj = __ldg(xl + k);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        const float kp = rhob * poly6_d(P, r2) * 2.0f;
        float3 rb = make_float3(kp * rx, kp * ry, kp * rz);
        if (r2 >= 1e-10f) {
            const float sg = spiky_scale(P, r2);
            const float3 ab = make_float3(k2 * rx * sg + gsb.x, k2 * ry * sg + gsb.y, k2 * rz * sg + gsb.z);
            const float3 r2b = grad_vjp(P, rx, ry, rz, r2, ab);
            rb.x += r2b.x;
            rb.y += r2b.y;
            rb.z += r2b.z;
        }
        own.x += rb.x;
        own.y += rb.y;
        own.z += rb.z;
        atomicAdd(gout + k, make_float4(-rb.x, -rb.y, -rb.z, 0.0f));
    });
    add_own(gout + s, own, 0.0f);
}

// ---- CS_PredictAndHash.glsl:102,114 reversed (slot -> particle order) ----------------------------
__global__ void k_ad_predict(uint32_t n, float dt, const uint32_t* __restrict__ ids, const float4* __restrict__ gx,
                             const float4* __restrict__ gv, const float4* __restrict__ x0b,
                             float4* __restrict__ posb, float4* __restrict__ velb)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t id = __ldg(ids + s);
        const float4 a = gx[s], v = gv[s], b = x0b[s];
        velb[id] = make_float4(v.x + dt * a.x, v.y + dt * a.y, v.z + dt * a.z, 0.0f);
        posb[id] = make_float4(a.x + b.x, a.y + b.y, a.z + b.z, 0.0f);
    }
}

// ---- launchers ---------------------------------------------------------------------------
static inline unsigned agrid(uint32_t n) { return (n + kAThreads - 1) / kAThreads; }

void launch_ad_lambda_rec(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                          const int2* table, const float4* xin, float4* xl, float4* auxl, float* rhol, cudaStream_t st)
{
    k_ad_lambda_rec<<<agrid(P.n), kAThreads, 0, st>>>(P, scenes, scene_of, order, table, xin, xl, auxl, rhol);
}

void launch_ad_deltap_rec(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                          const int2* table, const float4* xl, float4* xout, float4* auxd, cudaStream_t st)
{
    k_ad_deltap_rec<<<agrid(P.n), kAThreads, 0, st>>>(P, scenes, scene_of, order, table, xl, xout, auxd);
}

void launch_ad_vorticity(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                         const int2* table, const float4* spos, const float4* somega, const uint32_t* ids,
                         const float4* velb, float4* posb_s, float4* omb, cudaStream_t st)
{
    k_ad_vorticity<<<agrid(P.n), kAThreads, 0, st>>>(P, scenes, scene_of, order, table, spos, somega, ids, velb,
                                                      posb_s, omb);
}

void launch_ad_integrate(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                         const int2* table, const float4* xs, const float4* sv, const float4* cp_pos,
                         const uint32_t* ids, const float4* posb, const float4* velb, const float4* posb_s,
                         const float4* omb, const float4* somega, float4* gx, float4* gv, float4* x0b, float* tgrad,
                         cudaStream_t st)
{
    k_ad_integrate<<<agrid(P.n), kAThreads, 0, st>>>(P, scenes, scene_of, order, table, xs, sv, cp_pos, ids, posb,
                                                      velb, posb_s, omb, somega, gx, gv, x0b, tgrad);
}

void launch_ad_deltap(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                      const int2* table, const float4* xl, const float4* auxd, const float4* gin, float4* gout,
                      float* tgrad, cudaStream_t st)
{
    k_ad_deltap<<<agrid(P.n), kAThreads, 0, st>>>(P, scenes, scene_of, order, table, xl, auxd, gin, gout, tgrad);
}

void launch_ad_lambda(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                      const int2* table, const float4* xl, const float4* auxl, const float* rhol, float4* gout,
                      cudaStream_t st)
{
    k_ad_lambda<<<agrid(P.n), kAThreads, 0, st>>>(P, scenes, scene_of, order, table, xl, auxl, rhol, gout);
}

void launch_ad_predict(uint32_t n, float dt, const uint32_t* ids, const float4* gx, const float4* gv,
                       const float4* x0b, float4* posb, float4* velb, int sms, cudaStream_t st)
{
    const uint32_t want = (n + 255u) / 256u, cap = (uint32_t)sms * 8u;
    k_ad_predict<<<want < 1 ? 1 : (want > cap ? cap : want), 256, 0, st>>>(n, dt, ids, gx, gv, x0b, posb, velb);
}

}  // namespace pbf
