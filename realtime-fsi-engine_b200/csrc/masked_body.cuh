// masked_body.cuh — per-particle bodies of the neighbour passes, shared by
// the single-scene kernels (k_masked.cu, k_dense.cu), the multi-scene kernels
// (k_batch.cu, k_dense.cu) and the adjoint's recording passes (k_adjoint.cu),
// so that all of them run the same arithmetic on every pair.
//
// Each pass is a `*_core` function parameterised by a walker: walk(hit, body)
// calls body(k) for every candidate k with hit(r^2) true, in the reference's
// visiting order (CS_ComputeLambdas.glsl:126-150: 27 hashed buckets, z outer,
// x inner, bucket contents in sorted order, colliding buckets once per
// neighbour cell), where k indexes the position array X the core reads
// neighbours from.  The walkers: masked_walk below (the hashed buckets
// themselves) and the run and bucket walks of k_dense.cu (the same hits in
// the same order over the relabelled arrays).
//
// masked_walk: for each bucket, up to 8 candidates are loaded with
// independent predicated loads and reduced to an 8-bit mask of hits; the
// body then runs for the set bits in candidate order.
#pragma once

#include "pbf_internal.cuh"

namespace pbf {

constexpr int kChunk = 8;

template <class Hit, class Body>
__device__ __forceinline__ void masked_walk(const DevParams& P, const int2* __restrict__ table, uint32_t mask,
                                            const float4* __restrict__ X, float xi, float yi, float zi, int self,
                                            Hit&& hit, Body&& body)
{
    const int cx = cell_coord(xi, P.h), cy = cell_coord(yi, P.h), cz = cell_coord(zi, P.h);
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
        const uint32_t hz = (uint32_t)(cz + dz) * kP3;
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
            const uint32_t hyz = hz ^ ((uint32_t)(cy + dy) * kP2);
#pragma unroll 1
            for (int dx = -1; dx <= 1; ++dx) {
                const uint32_t hsh = (((uint32_t)(cx + dx) * kP1) ^ hyz) & mask;
                const int2 se = __ldg(table + hsh);
                if (se.x == -1) continue;
#pragma unroll 1
                for (int k0 = se.x; k0 < se.y; k0 += kChunk) {
                    uint32_t m = 0;
#pragma unroll
                    for (int c = 0; c < kChunk; ++c) {
                        const int k = k0 + c;
                        if (k < se.y) {
                            const float4 xj = __ldg(X + k);
                            const float rx = xi - xj.x, ry = yi - xj.y, rz = zi - xj.z;
                            const float r2 = rx * rx + ry * ry + rz * rz;
                            if (hit(r2) && k != self) m |= 1u << c;
                        }
                    }
                    while (m) {
                        const int c = __ffs(m) - 1;
                        m &= m - 1u;
                        body(k0 + c);
                    }
                }
            }
        }
    }
}

// Neighbour data sources of the pass cores: global memory through the
// read-only path, or plain loads (shared memory).
struct GSrc {
    const float4* __restrict__ p;
    __device__ __forceinline__ float4 operator[](int k) const { return __ldg(p + k); }
};
struct GMag {  // |omega| in the w of a float4 (omega, |omega|) array
    const float4* __restrict__ p;
    __device__ __forceinline__ float operator[](int k) const { return __ldg(&p[k].w); }
};
struct SSrc {
    const float4* p;
    __device__ __forceinline__ float4 operator[](int k) const { return p[k]; }
};
struct GMagX {  // |omega| in the w of a position array, read as the whole float4 the pair body loads anyway
    const float4* __restrict__ p;
    __device__ __forceinline__ float operator[](int k) const { return __ldg(p + k).w; }
};
struct SMagW {  // |omega| staged in the w of a position array
    const float4* p;
    __device__ __forceinline__ float operator[](int k) const { return p[k].w; }
};

// Walker over the hashed buckets of the sorted arrays (slot k = sorted slot).
struct HashWalk {
    const DevParams& P;
    const int2* table;
    uint32_t mask;
    const float4* X;
    float4 xi;
    int self;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        masked_walk(P, table, mask, X, xi.x, xi.y, xi.z, self, hit, body);
    }
};

// ---- CS_ComputeLambdas.glsl:108-162 -----------------------------------------------------------
// Returns (x*, lambda); also rho, grad C_i (the scaled sum of spiky
// gradients), the denominator sum |grad C|^2 + eps that lambda divides by
// (the adjoint replays them) and, in b_out, the part of the delta-p sum of
// CS_ComputeDeltaP.glsl:120-166 that does not depend on the neighbours'
// lambdas: lambda_i * sum_j gradW_ij + sum_j s_corr(r_ij) * gradW_ij (before
// the 1/rho0 scale).  The delta-p pass of the same iteration, over the same
// positions and pairs, then adds only sum_j lambda_j * gradW_ij.
template <class XS, class Walk>
__device__ __forceinline__ float4 lambda_core(const DevParams& P, XS X, float4 xi, Walk&& walk, float& rho_out,
                                              float3& g_out, float& den_out, float3& b_out)
{
    // s_corr = -k (W / W(dq))^n per pair: the pair body sums (W / W(dq))^n *
    // gradW, the factor -k is applied once after the walk
    const bool scorr = P.scorr && P.wq > 1e-12f;
    float rho = P.w0_self, sg = 0.f, gz = 0.f, sz = 0.f;
    float2 gxy = make_float2(0.f, 0.f), sxy = make_float2(0.f, 0.f);
    const float2 xyi = make_float2(xi.x, xi.y);
    walk([&](float r2) { return r2 <= P.h2; },
         [&](int k) {
             const float4 xj = X[k];
             const float2 rxy = sub_f32x2(xyi, make_float2(xj.x, xj.y));
             const float rx = rxy.x, ry = rxy.y, rz = xi.z - xj.z;
             const float r2 = rx * rx + ry * ry + rz * rz;
             const float w = poly6_in(P, r2);
             rho += w;
             if (r2 >= 1e-10f) {
                 const float sc = spiky_scale(P, r2);
                 const float2 axy = mul_f32x2(rxy, sc);
                 const float ax = axy.x, ay = axy.y, az = rz * sc;
                 sg += ax * ax + ay * ay + az * az;
                 gxy = add_f32x2(gxy, axy);
                 gz += az;
                 if (scorr) {
                     const float ratio = w * P.inv_wq;
                     float pw;
                     if (P.ncorr_is4) {
                         const float q = ratio * ratio;
                         pw = q * q;
                     } else {
                         pw = powf(ratio, P.n_corr);
                     }
                     sxy = fma_f32x2(axy, pw, sxy);
                     sz = __fmaf_rn(az, pw, sz);
                 }
             }
         });
    const float lam_gx = gxy.x, lam_gy = gxy.y, lam_gz = gz;  // sum_j gradW_ij, unscaled
    float gx = gxy.x, gy = gxy.y;
    gx *= P.inv_rho0;
    gy *= P.inv_rho0;
    gz *= P.inv_rho0;
    const float C = fmaxf(rho / P.rho0 - 1.0f, -P.cohesion);
    sg = sg * P.inv_rho0_sq + (gx * gx + gy * gy + gz * gz);
    rho_out = rho;
    g_out = make_float3(gx, gy, gz);
    den_out = sg + P.eps;
    const float lam = -C / den_out;
    const float kc = scorr ? -P.k_corr : 0.f;
    b_out = make_float3(__fmaf_rn(lam, lam_gx, kc * sxy.x), __fmaf_rn(lam, lam_gy, kc * sxy.y),
                        __fmaf_rn(lam, lam_gz, kc * sz));
    return make_float4(xi.x, xi.y, xi.z, lam);
}

__device__ __forceinline__ float4 lambda_particle_x(const DevParams& P, const int2* __restrict__ table,
                                                    uint32_t mask, const float4* __restrict__ xin, int s,
                                                    float& rho_out, float3& g_out, float& den_out)
{
    const float4 xi = __ldg(xin + s);
    float3 b;
    const float4 out = lambda_core(P, GSrc{xin}, xi, HashWalk{P, table, mask, xin, xi, s}, rho_out, g_out, den_out, b);
    P.dpb[s] = make_float4(b.x, b.y, b.z, 0.f);
    return out;
}

__device__ __forceinline__ float4 lambda_particle(const DevParams& P, const int2* __restrict__ table, uint32_t mask,
                                                  const float4* __restrict__ xin, int s, float& rho_out)
{
    float3 g;
    float den;
    return lambda_particle_x(P, table, mask, xin, s, rho_out, g, den);
}

// s_corr * (poly6 coefficient form) of CS_ComputeDeltaP.glsl:94-104 added to
// lambda_i + lambda_j; valid for r2 < h2 (the adjoint's reverse delta-p pass
// differentiates it per pair).
__device__ __forceinline__ float scorr_term(const DevParams& P, float r2)
{
    const float d = P.h2 - r2;
    const float w = P.poly6 * d * d * d;
    if (P.wq > 1e-12f && w > 0.0f) {
        const float ratio = w * P.inv_wq;
        float pw;
        if (P.ncorr_is4) {
            const float q = ratio * ratio;
            pw = q * q;
        } else {
            pw = powf(ratio, P.n_corr);
        }
        return -P.k_corr * pw;
    }
    return 0.0f;
}

// ---- CS_ComputeDeltaP.glsl:120-166 + CS_ApplyDeltaP.glsl:80-124 --------------------------------
// Returns (x* + dp, lambda); dp_raw = dp before the 0.5 h clamp.  b is the
// lambda pass's b_out for this particle: the shader's per-pair factor
// (lambda_i + lambda_j + s_corr) * gradW_ij is summed as b + sum_j lambda_j *
// gradW_ij, so the pair body here loads and scales only lambda_j.
template <class XS, class Walk>
__device__ __forceinline__ float4 deltap_core(const DevParams& P, const SdfDev& sdf, XS X, float4 xi, Walk&& walk,
                                              float3& dp_raw, float3 b)
{
    const float li = xi.w;
    float dz = b.z;
    float2 dxy = make_float2(b.x, b.y);
    const float2 xyi = make_float2(xi.x, xi.y);
    walk([&](float r2) { return r2 <= P.h2 && r2 >= 1e-10f; },
         [&](int k) {
             const float4 xj = X[k];
             const float2 rxy = sub_f32x2(xyi, make_float2(xj.x, xj.y));
             const float rx = rxy.x, ry = rxy.y, rz = xi.z - xj.z;
             const float r2 = rx * rx + ry * ry + rz * rz;
             const float g = spiky_scale(P, r2) * xj.w;
             dxy = fma_f32x2(rxy, g, dxy);
             dz = __fmaf_rn(rz, g, dz);
         });
    float dx = dxy.x, dy = dxy.y;
    // rounded products (not fused into the x + dp below)
    dx = __fmul_rn(dx, P.inv_rho0);
    dy = __fmul_rn(dy, P.inv_rho0);
    dz = __fmul_rn(dz, P.inv_rho0);
    dp_raw = make_float3(dx, dy, dz);
    const float l2 = dx * dx + dy * dy + dz * dz;
    if (l2 > P.max_dp * P.max_dp) {
        const float sc = P.max_dp * rsqrtf(l2);
        dx = __fmul_rn(dx, sc);
        dy = __fmul_rn(dy, sc);
        dz = __fmul_rn(dz, sc);
    }
    float3 p = make_float3(xi.x + dx, xi.y + dy, xi.z + dz);
    if (sdf.enabled) {
        float3 nrm;
        sdf_project(sdf, p, nrm);
    }
    return make_float4(p.x, p.y, p.z, li);
}

__device__ __forceinline__ float4 deltap_particle_x(const DevParams& P, const int2* __restrict__ table,
                                                    uint32_t mask, const SdfDev& sdf,
                                                    const float4* __restrict__ xin, int s, float3& dp_raw)
{
    const float4 xi = __ldg(xin + s);
    const float4 b = __ldg(P.dpb + s);
    return deltap_core(P, sdf, GSrc{xin}, xi, HashWalk{P, table, mask, xin, xi, s}, dp_raw,
                       make_float3(b.x, b.y, b.z));
}

__device__ __forceinline__ float4 deltap_particle(const DevParams& P, const int2* __restrict__ table, uint32_t mask,
                                                  const SdfDev& sdf, const float4* __restrict__ xin, int s)
{
    float3 dp;
    return deltap_particle_x(P, table, mask, sdf, xin, s, dp);
}

// ---- CS_Integrate.glsl:135-280 (pre-dispatch neighbour velocities) ---------------------------
// From x* (x4), the predicted velocity v0, the substep start p0 and the
// neighbours' (X, V): the committed position xo (w = p0.w), velocity vo
// (w = v0.w) and, when vorticity is on, omega4 = (omega, |omega|).
template <class XS, class VS, class P0, class Walk>
__device__ __forceinline__ void integrate_core(const DevParams& P, const float* bmin, const float* bmax,
                                               const SdfDev& sdf, XS X, VS V, float4 x4, float4 v0, P0&& p0_load,
                                               Walk&& walk, float4& xo, float4& vo, float4& omega4)
{
    float fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    float2 fxy = make_float2(0.f, 0.f);
    const float2 xyi = make_float2(x4.x, x4.y), vxy0 = make_float2(v0.x, v0.y);
    if (P.visc_on || P.vort_on) {
        walk([&](float r2) { return r2 <= P.h2; },
             [&](int k) {
                 const float4 xj = X[k];
                 const float2 rxy = sub_f32x2(xyi, make_float2(xj.x, xj.y));
                 const float rx = rxy.x, ry = rxy.y, rz = x4.z - xj.z;
                 const float r2 = rx * rx + ry * ry + rz * rz;
                 const float4 vj = V[k];
                 const float2 uxy = sub_f32x2(make_float2(vj.x, vj.y), vxy0);
                 const float ux = uxy.x, uy = uxy.y, uz = vj.z - v0.z;
                 if (P.visc_on) {
                     const float w = poly6_in(P, r2) * P.inv_rho0;
                     fxy = fma_f32x2(uxy, w, fxy);
                     fz = __fmaf_rn(uz, w, fz);
                 }
                 if (P.vort_on && r2 >= 1e-10f) {
                     const float sc = spiky_scale(P, r2);
                     const float2 axy = mul_f32x2(rxy, sc);
                     const float ax = axy.x, ay = axy.y, az = rz * sc;
                     // a*b - c*d with the rounding fixed (one product rounded,
                     // one fused), so every instantiation gives the same bits
                     cx += __fmaf_rn(uy, az, -__fmul_rn(uz, ay));
                     cy += __fmaf_rn(uz, ax, -__fmul_rn(ux, az));
                     cz += __fmaf_rn(ux, ay, -__fmul_rn(uy, ax));
                 }
             });
    }
    // the substep-start position is needed only now: loaded after the walk,
    // it holds no registers across it
    const float4 p0 = p0_load();
    const float fx = fxy.x, fy = fxy.y;
    float3 x = make_float3(x4.x, x4.y, x4.z);
    float vdx = 0.f, vdy = 0.f, vdz = 0.f;
    if (P.visc_on) {
        vdx = __fmul_rn(fx, P.viscosity);
        vdy = __fmul_rn(fy, P.viscosity);
        vdz = __fmul_rn(fz, P.viscosity);
    }
    if (P.vort_on) {
        const float ox = cx * P.inv_rho0, oy = cy * P.inv_rho0, oz = cz * P.inv_rho0;
        omega4 = make_float4(ox, oy, oz, sqrtf(ox * ox + oy * oy + oz * oz));
    }
    bool colx = false, coly = false, colz = false;
    if (x.x <= bmin[0]) { x.x = bmin[0]; colx = true; }
    if (x.x >= bmax[0]) { x.x = bmax[0]; colx = true; }
    if (x.y <= bmin[1]) { x.y = bmin[1]; coly = true; }
    if (x.y >= bmax[1]) { x.y = bmax[1]; coly = true; }
    if (x.z <= bmin[2]) { x.z = bmin[2]; colz = true; }
    if (x.z >= bmax[2]) { x.z = bmax[2]; colz = true; }
    bool col_sdf = false;
    float3 nrm = make_float3(0.0f, 0.0f, 0.0f);
    if (sdf.enabled) col_sdf = sdf_project(sdf, x, nrm);
    float vx = __fmaf_rn(x.x - p0.x, P.inv_dt, vdx);
    float vy = __fmaf_rn(x.y - p0.y, P.inv_dt, vdy);
    float vz = __fmaf_rn(x.z - p0.z, P.inv_dt, vdz);
    const float sp2 = vx * vx + vy * vy + vz * vz;
    if (sp2 > 2500.0f) {
        const float sc = 50.0f / sqrtf(sp2);
        vx *= sc;
        vy *= sc;
        vz *= sc;
    }
    if (colx) vx *= -P.damping;
    if (coly) vy *= -P.damping;
    if (colz) vz *= -P.damping;
    if (col_sdf) {
        const float vn = vx * nrm.x + vy * nrm.y + vz * nrm.z;
        vx -= vn * nrm.x;
        vy -= vn * nrm.y;
        vz -= vn * nrm.z;
    }
    xo = make_float4(x.x, x.y, x.z, p0.w);
    vo = make_float4(vx, vy, vz, v0.w);
}

// Commits x and v of slot s: writes pos/vel at the particle id, sx0[s] = x
// and somega[s] = (omega, |omega|).
__device__ __forceinline__ void integrate_particle(const DevParams& P, const int2* __restrict__ table, uint32_t mask,
                                                   const float* bmin, const float* bmax, const SdfDev& sdf,
                                                   const float4* __restrict__ xs, const float4* __restrict__ sv,
                                                   float4* __restrict__ sx0, float4* __restrict__ somega,
                                                   const uint32_t* __restrict__ ids, float4* __restrict__ pos,
                                                   float4* __restrict__ vel, int s)
{
    const float4 x4 = __ldg(xs + s);
    const float4 v0 = __ldg(sv + s);
    float4 xo, vo, om;
    integrate_core(P, bmin, bmax, sdf, GSrc{xs}, GSrc{sv}, x4, v0, [&] { return sx0[s]; },
                   HashWalk{P, table, mask, xs, x4, s}, xo, vo, om);
    if (P.vort_on) somega[s] = om;
    const uint32_t id = __ldg(ids + s);
    pos[id] = xo;
    vel[id] = vo;
    sx0[s] = xo;
}

// ---- CS_VorticityConfinement.glsl:133-167 (pass 1) ----------------------------------------------
// Velocity increment eps (N x omega_i) dt of a particle at xi with vorticity
// w; returns false when |eta| < 1e-6 (no change).
// MS: source of the neighbours' |omega| (MS[k] -> float).
template <class XS, class MS, class WL, class Walk>
__device__ __forceinline__ bool vorticity_core(const DevParams& P, XS X, MS OMAG, float4 xi, WL&& w_load, Walk&& walk,
                                               float3& dv)
{
    float ez = 0.f;
    float2 exy = make_float2(0.f, 0.f);
    const float2 xyi = make_float2(xi.x, xi.y);
    walk([&](float r2) { return r2 <= P.h2 && r2 >= 1e-10f; },
         [&](int k) {
             const float4 xj = X[k];
             const float2 rxy = sub_f32x2(xyi, make_float2(xj.x, xj.y));
             const float rx = rxy.x, ry = rxy.y, rz = xi.z - xj.z;
             const float r2 = rx * rx + ry * ry + rz * rz;
             const float sc = spiky_scale(P, r2) * OMAG[k];
             exy = fma_f32x2(rxy, sc, exy);
             ez = __fmaf_rn(rz, sc, ez);
         });
    float ex = exy.x, ey = exy.y;
    ex *= P.inv_rho0;
    ey *= P.inv_rho0;
    ez *= P.inv_rho0;
    const float el = sqrtf(ex * ex + ey * ey + ez * ez);
    if (el < 1e-6f) return false;
    const float4 w = w_load();  // the particle's own omega, loaded after the walk
    const float nx = ex / el, ny = ey / el, nz = ez / el;
    const float crx = __fmaf_rn(ny, w.z, -__fmul_rn(nz, w.y)), cry = __fmaf_rn(nz, w.x, -__fmul_rn(nx, w.z)),
                crz = __fmaf_rn(nx, w.y, -__fmul_rn(ny, w.x));
    // rounded products: the caller adds dv to v, and a fused multiply-add
    // there would round differently from one kernel to another
    dv = make_float3(__fmul_rn(P.vort_eps * crx, P.dt), __fmul_rn(P.vort_eps * cry, P.dt),
                     __fmul_rn(P.vort_eps * crz, P.dt));
    return true;
}

__device__ __forceinline__ void vorticity_particle(const DevParams& P, const int2* __restrict__ table, uint32_t mask,
                                                   const float4* __restrict__ spos,
                                                   const float4* __restrict__ somega,
                                                   const uint32_t* __restrict__ ids, float4* __restrict__ vel, int s)
{
    const float4 xi = __ldg(spos + s);
    float3 dv;
    if (!vorticity_core(P, GSrc{spos}, GMag{somega}, xi, [&] { return __ldg(somega + s); },
                        HashWalk{P, table, mask, spos, xi, s}, dv))
        return;
    const uint32_t id = __ldg(ids + s);
    float4 v = vel[id];
    v.x += dv.x;
    v.y += dv.y;
    v.z += dv.z;
    vel[id] = v;
}

}  // namespace pbf
