// pbf_internal.cuh — shared device-side definitions of the B200 PBF engine.
//
// Data layout in HBM (one handle = one scene):
//   particle order (the caller's indices, as the reference keeps them):
//     pos4[N], vel4[N]        float4, w carries the Particle pad word
//     keys[N]                 u32 hash key of the predicted position
//   sorted order (slot s = rank of particle ids[s] in the stable (key, id) sort):
//     skeys[N], ids[N]        sorted keys and the particle id of every slot
//     sx[2][N]                float4 (x*, lambda), Jacobi ping-pong
//     sv[N]                   float4 (v after gravity, pad2)
//     sx0[N]                  float4 (x at substep start, pad0); integrate
//                             overwrites it with the committed x for the
//                             vorticity pass
//     somega[N]               float4 (omega = curl / rho0, |omega|)
//     rho[N]                  float density of the last lambda pass
//   table[H]                  int2 (start, end) of each hash bucket in sorted
//                             order, (-1, -1) when empty
// Every neighbour pass reads its candidates from contiguous sorted slots, so a
// bucket of ~8 particles is one 128-byte run of float4 instead of the
// reference's two dependent scattered loads per candidate.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pbf {

// getGridHash primes (CS_PredictAndHash.glsl:77-83); int wrap-around
// arithmetic is reproduced with unsigned multiplication.
constexpr uint32_t kP1 = 73856093u;
constexpr uint32_t kP2 = 19349663u;
constexpr uint32_t kP3 = 83492791u;

struct SdfDev {
    const float* dist;      // index(x,y,z) = (x*dy + y)*dz + z
    const float* slab_min;  // 6 floats: min over faces x=0, x=dx-1, y=0, y=dy-1, z=0, z=dz-1
    int dx, dy, dz;
    float ox, oy, oz;
    float cell, inv_cell;
    float padding;
    int containment;
    int enabled;
};

// Kernel-side constants: the FluidConfigUBO block (PBFluids.h:21-61) plus the
// per-dispatch uniforms of PBFluids::step, passed by value (constant bank).
struct DevParams {
    float bmin[3], bmax[3];
    float g[3];
    float dt;        // substep dt
    float inv_dt;    // (dt > 0) ? 1/dt : 0   (CS_Integrate.glsl:244)
    float h, h2;
    float rho0, inv_rho0, inv_rho0_sq;
    float eps, wq, inv_wq, k_corr, n_corr;
    float viscosity, damping, cohesion;
    float w0_self, poly6, spiky;
    float max_dp;    // 0.5 h (CS_ApplyDeltaP.glsl:92)
    uint32_t mask;
    uint32_t n;
    uint32_t scorr, visc_on, vort_on, apbf;
    uint32_t ncorr_is4;
    float vort_eps;
    uint32_t interacting;
    float ipos[3];
    float i_radius, i_strength;
    float cam[3];
    float lod_max_dist;
    uint32_t min_lod, max_lod;
    SdfDev sdf;
    // per particle, indexed as the position arrays of the solver iterations:
    // the lambda-independent part of the delta-p sum, written by each lambda
    // pass and read by the delta-p pass of the same iteration (masked_body.cuh)
    float4* dpb;
};

__device__ __forceinline__ uint32_t grid_hash(int cx, int cy, int cz, uint32_t mask)
{
    return (((uint32_t)cx * kP1) ^ ((uint32_t)cy * kP2) ^ ((uint32_t)cz * kP3)) & mask;
}

// ivec3(floor(x / h)) with an IEEE-rounded FP32 division, as the shader.
__device__ __forceinline__ int cell_coord(float x, float h) { return (int)floorf(__fdiv_rn(x, h)); }

// Predict step of CS_PredictAndHash.glsl:98-114, written with explicit
// intrinsics so that every kernel that re-derives x* from (pos, vel) gets the
// same bits (the predict/hash kernel and the reorder kernel both call it).
__device__ __forceinline__ void predict_particle(const DevParams& P, float4 p, float4 v, float3& vp, float3& xs)
{
    float vx = __fmaf_rn(P.g[0], P.dt, v.x);
    float vy = __fmaf_rn(P.g[1], P.dt, v.y);
    float vz = __fmaf_rn(P.g[2], P.dt, v.z);
    if (P.interacting) {
        const float tx = __fsub_rn(P.ipos[0], p.x);
        const float ty = __fsub_rn(P.ipos[1], p.y);
        const float tz = __fsub_rn(P.ipos[2], p.z);
        const float dist = __fsqrt_rn(__fmaf_rn(tz, tz, __fmaf_rn(ty, ty, __fmul_rn(tx, tx))));
        if (dist < P.i_radius && dist > 1e-5f) {
            const float falloff = __fsub_rn(1.0f, __fdiv_rn(dist, P.i_radius));
            const float s = __fmul_rn(__fmul_rn(__fdiv_rn(P.i_strength, dist), falloff), P.dt);
            vx = __fmaf_rn(tx, s, vx);
            vy = __fmaf_rn(ty, s, vy);
            vz = __fmaf_rn(tz, s, vz);
        }
    }
    vp = make_float3(vx, vy, vz);
    xs = make_float3(__fmaf_rn(vx, P.dt, p.x), __fmaf_rn(vy, P.dt, p.y), __fmaf_rn(vz, P.dt, p.z));
}

// poly6 (CS_ComputeLambdas.glsl:74-81), valid for r2 <= h2.
__device__ __forceinline__ float poly6_in(const DevParams& P, float r2)
{
    const float d = P.h2 - r2;
    return P.poly6 * d * d * d;
}

// Packed FP32 pairs (sm_100 f32x2 instructions): each lane is rounded exactly
// as the scalar operation, so a pair computed this way has the scalar bits.
__device__ __forceinline__ uint64_t f32x2_pack(float2 a)
{
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 f32x2_unpack(uint64_t r)
{
    float2 o;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(o.x), "=f"(o.y) : "l"(r));
    return o;
}
// a - b
__device__ __forceinline__ float2 sub_f32x2(float2 a, float2 b)
{
    uint64_t r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f32x2_pack(a)), "l"(f32x2_pack(b)));
    return f32x2_unpack(r);
}
// a + b
__device__ __forceinline__ float2 add_f32x2(float2 a, float2 b)
{
    uint64_t r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f32x2_pack(a)), "l"(f32x2_pack(b)));
    return f32x2_unpack(r);
}
// a * s
__device__ __forceinline__ float2 mul_f32x2(float2 a, float s)
{
    uint64_t r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f32x2_pack(a)), "l"(f32x2_pack(make_float2(s, s))));
    return f32x2_unpack(r);
}
// a * s + c, fused
__device__ __forceinline__ float2 fma_f32x2(float2 a, float s, float2 c)
{
    uint64_t r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;"
        : "=l"(r)
        : "l"(f32x2_pack(a)), "l"(f32x2_pack(make_float2(s, s))), "l"(f32x2_pack(c)));
    return f32x2_unpack(r);
}

// spiky gradient scalar factor (CS_ComputeLambdas.glsl:83-92): grad = r * s,
// valid for 1e-10 <= r2 <= h2.  -spiky (h - |r|)^2 / |r| evaluated with one
// reciprocal square root (|r| = r2 * rsqrt(r2)) instead of a square root and
// a division; the difference is FP32 rounding.
__device__ __forceinline__ float spiky_scale(const DevParams& P, float r2)
{
    const float inv = rsqrtf(r2);
    const float diff = P.h - r2 * inv;
    return -P.spiky * diff * diff * inv;
}

// computeSCorr (CS_ComputeDeltaP.glsl:94-104), valid for r2 < h2 (w > 0).
__device__ __forceinline__ float scorr_in(const DevParams& P, float r2)
{
    if (!P.scorr) return 0.0f;
    const float w = poly6_in(P, r2);
    if (P.wq <= 1e-12f || w <= 0.0f) return 0.0f;
    const float ratio = w / P.wq;
    if (ratio <= 0.0f) return 0.0f;
    float pw;
    if (P.ncorr_is4) {
        const float r2_ = ratio * ratio;
        pw = r2_ * r2_;
    } else {
        pw = powf(ratio, P.n_corr);
    }
    return -P.k_corr * pw;
}

// ---- SDF grid sampling (software trilinear, clamp to edge) -----------------
__device__ __forceinline__ float sdf_texel(const SdfDev& S, int x, int y, int z)
{
    return __ldg(S.dist + ((long)x * S.dy + y) * S.dz + z);
}

// texture(sdfTexture, ((p - o)/cell + 0.5)/dims).r with GL_LINEAR and
// CLAMP_TO_EDGE (CS_Integrate.glsl:86-89): texel-space u = (p - o)/cell.
__device__ __forceinline__ float sdf_sample(const SdfDev& S, float px, float py, float pz)
{
    float u = (px - S.ox) * S.inv_cell;
    float v = (py - S.oy) * S.inv_cell;
    float w = (pz - S.oz) * S.inv_cell;
    u = fminf(fmaxf(u, 0.0f), (float)(S.dx - 1));
    v = fminf(fmaxf(v, 0.0f), (float)(S.dy - 1));
    w = fminf(fmaxf(w, 0.0f), (float)(S.dz - 1));
    const float fu = floorf(u), fv = floorf(v), fw = floorf(w);
    const int i0 = (int)fu, j0 = (int)fv, k0 = (int)fw;
    const int i1 = min(i0 + 1, S.dx - 1), j1 = min(j0 + 1, S.dy - 1), k1 = min(k0 + 1, S.dz - 1);
    const float a = u - fu, b = v - fv, c = w - fw;
    const float c000 = sdf_texel(S, i0, j0, k0), c001 = sdf_texel(S, i0, j0, k1);
    const float c010 = sdf_texel(S, i0, j1, k0), c011 = sdf_texel(S, i0, j1, k1);
    const float c100 = sdf_texel(S, i1, j0, k0), c101 = sdf_texel(S, i1, j0, k1);
    const float c110 = sdf_texel(S, i1, j1, k0), c111 = sdf_texel(S, i1, j1, k1);
    const float c00 = c000 + (c001 - c000) * c, c01 = c010 + (c011 - c010) * c;
    const float c10 = c100 + (c101 - c100) * c, c11 = c110 + (c111 - c110) * c;
    const float c0 = c00 + (c01 - c00) * b, c1 = c10 + (c11 - c10) * b;
    return c0 + (c1 - c0) * a;
}

// True when no obstacle projection can happen at p: p lies more than one and
// a half cells outside the grid on an axis whose boundary face holds only
// values >= padding, so all seven samples of the projection read that face
// (clamp to edge) and d >= padding.  Exact skip, obstacle mode only.
__device__ __forceinline__ bool sdf_far_obstacle(const SdfDev& S, float px, float py, float pz)
{
    if (S.containment) return false;
    const float u = (px - S.ox) * S.inv_cell;
    const float v = (py - S.oy) * S.inv_cell;
    const float w = (pz - S.oz) * S.inv_cell;
    if (u < -1.5f && __ldg(S.slab_min + 0) >= S.padding) return true;
    if (u > (float)S.dx + 0.5f && __ldg(S.slab_min + 1) >= S.padding) return true;
    if (v < -1.5f && __ldg(S.slab_min + 2) >= S.padding) return true;
    if (v > (float)S.dy + 0.5f && __ldg(S.slab_min + 3) >= S.padding) return true;
    if (w < -1.5f && __ldg(S.slab_min + 4) >= S.padding) return true;
    if (w > (float)S.dz + 0.5f && __ldg(S.slab_min + 5) >= S.padding) return true;
    return false;
}

// Obstacle / container projection (CS_ApplyDeltaP.glsl:108-121 and
// CS_Integrate.glsl:216-240).  Returns true on contact with the push normal.
__device__ __forceinline__ bool sdf_project(const SdfDev& S, float3& p, float3& nrm)
{
    if (sdf_far_obstacle(S, p.x, p.y, p.z)) return false;
    const float e = S.cell;
    const float d = sdf_sample(S, p.x, p.y, p.z);
    // no contact whatever the gradient: skip its six samples
    if (S.containment ? !(d > -S.padding) : !(d < S.padding)) return false;
    const float inv2e = 1.0f / (2.0f * e);
    const float gx = (sdf_sample(S, p.x + e, p.y, p.z) - sdf_sample(S, p.x - e, p.y, p.z)) * inv2e;
    const float gy = (sdf_sample(S, p.x, p.y + e, p.z) - sdf_sample(S, p.x, p.y - e, p.z)) * inv2e;
    const float gz = (sdf_sample(S, p.x, p.y, p.z + e) - sdf_sample(S, p.x, p.y, p.z - e)) * inv2e;
    const float len = sqrtf(gx * gx + gy * gy + gz * gz);
    if (!(len > 1e-6f)) return false;
    if (S.containment) {
        if (d > -S.padding) {
            nrm = make_float3(-gx / len, -gy / len, -gz / len);
            const float s = d + S.padding;
            p = make_float3(p.x + nrm.x * s, p.y + nrm.y * s, p.z + nrm.z * s);
            return true;
        }
    } else {
        if (d < S.padding) {
            nrm = make_float3(gx / len, gy / len, gz / len);
            const float s = S.padding - d;
            p = make_float3(p.x + nrm.x * s, p.y + nrm.y * s, p.z + nrm.z * s);
            return true;
        }
    }
    return false;
}

// The 27-bucket neighbour walk shared by every neighbour pass, in the
// reference's order (z outer, x inner; CS_ComputeLambdas.glsl:126-150).
// `body(k)` is called for every slot k of every non-empty bucket except the
// particle's own slot; colliding buckets are walked once per neighbour cell.
template <class Body>
__device__ __forceinline__ void for_each_neighbour(const DevParams& P, const int2* __restrict__ table, float xi,
                                                   float yi, float zi, int self, Body&& body)
{
    const int cx = cell_coord(xi, P.h), cy = cell_coord(yi, P.h), cz = cell_coord(zi, P.h);
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
        const uint32_t hz = (uint32_t)(cz + dz) * kP3;
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
            const uint32_t hyz = hz ^ ((uint32_t)(cy + dy) * kP2);
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const uint32_t hsh = (((uint32_t)(cx + dx) * kP1) ^ hyz) & P.mask;
                const int2 se = __ldg(table + hsh);
                if (se.x == -1) continue;
                for (int k = se.x; k < se.y; ++k) {
                    if (k == self) continue;
                    body(k);
                }
            }
        }
    }
}

}  // namespace pbf
