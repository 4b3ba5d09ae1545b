// k_queue.cu — neighbour passes with per-lane pair queues (thread per
// particle, Morton order).
//
// About 15% of the ~216 candidates a particle visits lie within h.  When the
// in-range body runs inside the candidate loop, a warp executes it for every
// candidate step on which any lane is in range — nearly all of them — with a
// few lanes active.  Here every lane runs a flat walk over its 27 buckets
// (one candidate per step, uniform trip structure across the warp), pushes
// in-range pairs into a small ring in shared memory, and the warp drains the
// rings one entry per lane only when most lanes hold work (or a ring is
// full, or the walks are over).  The body then runs at near full width.
//
// Each particle still visits exactly the reference's candidate multiset (its
// current cell's 27 hashed buckets, self excluded); only the FP32 summation
// order differs from the sequential loop.
#include "pbf_kernels.h"

namespace pbf {

constexpr int kQThreads = 128;
constexpr int kQDepth = 8;  // ring entries per lane (power of two)

// Walk state over the 27 buckets of one cell, z outer / x inner
// (CS_ComputeLambdas.glsl:126-150).
struct BucketWalk {
    int cx, cy, cz;
    int b;     // next bucket index 0..27
    int k, e;  // current slot range
    int self;

    __device__ __forceinline__ void init(const DevParams& P, float x, float y, float z, int s)
    {
        cx = cell_coord(x, P.h);
        cy = cell_coord(y, P.h);
        cz = cell_coord(z, P.h);
        b = 0;
        k = 0;
        e = 0;
        self = s;
    }

    __device__ __forceinline__ bool next(const DevParams& P, const int2* __restrict__ table, int& out)
    {
        for (;;) {
            while (k >= e) {
                if (b >= 27) return false;
                const int dz = b / 9 - 1, dy = (b / 3) % 3 - 1, dx = b % 3 - 1;
                ++b;
                const uint32_t hsh = grid_hash(cx + dx, cy + dy, cz + dz, P.mask);
                const int2 se = __ldg(table + hsh);
                if (se.x == -1) continue;
                k = se.x;
                e = se.y;
            }
            const int c = k++;
            if (c != self) {
                out = c;
                return true;
            }
        }
    }
};

// Drain policy: a round when at least 3/4 of the warp holds an entry, when a
// ring is full, or unconditionally once no lane is walking any more.
__device__ __forceinline__ bool drain_now(bool walking_any, unsigned has_mask, bool any_full)
{
    return any_full || __popc(has_mask) >= 24 || (!walking_any && has_mask != 0u);
}

// Generic queued walk.  test(k, entry&) decides whether candidate k is kept
// and fills its ring entry; use(entry) consumes one entry.
template <class Test, class Use>
__device__ __forceinline__ void queued_walk(const DevParams& P, const int2* __restrict__ table, bool active, float x,
                                            float y, float z, int self, float4* ring, Test&& test, Use&& use)
{
    BucketWalk W;
    W.init(P, x, y, z, self);
    int qh = 0, qt = 0;
    bool walking = active;
    for (;;) {
        int k = 0;
        if (walking) walking = W.next(P, table, k);
        if (walking) {
            float4 ent;
            if (test(k, ent)) {
                ring[(qh & (kQDepth - 1)) * kQThreads] = ent;
                ++qh;
            }
        }
        const bool walking_any = __any_sync(0xffffffffu, walking);
        for (;;) {
            const bool has = qh > qt;
            const unsigned has_mask = __ballot_sync(0xffffffffu, has);
            const bool any_full = __any_sync(0xffffffffu, qh - qt >= kQDepth);
            if (!drain_now(walking_any, has_mask, any_full)) break;
            if (has) {
                use(ring[(qt & (kQDepth - 1)) * kQThreads]);
                ++qt;
            }
        }
        if (!walking_any) break;
    }
}

// ---- CS_ComputeLambdas.glsl:108-162 ------------------------------------------------------
__global__ void __launch_bounds__(kQThreads) k_lambda_q(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, float* __restrict__ rho_out,
                                                        const int2* __restrict__ table, const uint32_t* __restrict__ lod,
                                                        uint32_t iter, const uint32_t* __restrict__ order)
{
    __shared__ float4 rings[kQDepth * kQThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (order ? (int)__ldg(order + t) : t) : -1;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    bool active = in;
    if (in) {
        xi = __ldg(xin + s);
        if (P.apbf && __ldg(lod + s) < iter) {
            xout[s] = xi;
            active = false;
        }
    }
    float rho = P.w0_self, sg = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    queued_walk(
        P, table, active, xi.x, xi.y, xi.z, s, rings + threadIdx.x,
        [&](int k, float4& ent) {
            const float4 xj = __ldg(xin + k);
            const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            ent = make_float4(rx, ry, rz, r2);
            return r2 <= P.h2;
        },
        [&](const float4& en) {
            const float r2 = en.w;
            rho += poly6_in(P, r2);
            if (r2 >= 1e-10f) {
                const float sc = spiky_scale(P, r2);
                const float ax = en.x * sc, ay = en.y * sc, az = en.z * sc;
                sg += (ax * ax + ay * ay + az * az) * P.inv_rho0_sq;
                gx += ax;
                gy += ay;
                gz += az;
            }
        });
    if (!active) return;
    gx *= P.inv_rho0;
    gy *= P.inv_rho0;
    gz *= P.inv_rho0;
    const float C = fmaxf(rho / P.rho0 - 1.0f, -P.cohesion);
    sg += gx * gx + gy * gy + gz * gz;
    xout[s] = make_float4(xi.x, xi.y, xi.z, -C / (sg + P.eps));
    rho_out[s] = rho;
}

// ---- CS_ComputeDeltaP.glsl:120-166 + CS_ApplyDeltaP.glsl:80-124 ------------------------------
__global__ void __launch_bounds__(kQThreads) k_deltap_q(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, const int2* __restrict__ table,
                                                        const uint32_t* __restrict__ lod, uint32_t iter,
                                                        const uint32_t* __restrict__ order)
{
    __shared__ float4 rings[kQDepth * kQThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (order ? (int)__ldg(order + t) : t) : -1;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    bool active = in;
    if (in) {
        xi = __ldg(xin + s);
        if (P.apbf && __ldg(lod + s) < iter) {
            xout[s] = xi;
            active = false;
        }
    }
    const float li = xi.w;
    float dx = 0.f, dy = 0.f, dz = 0.f;
    queued_walk(
        P, table, active, xi.x, xi.y, xi.z, s, rings + threadIdx.x,
        [&](int k, float4& ent) {
            const float4 xj = __ldg(xin + k);
            const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            ent = make_float4(rx, ry, rz, xj.w);
            return r2 <= P.h2 && r2 >= 1e-10f;
        },
        [&](const float4& en) {
            const float r2 = en.x * en.x + en.y * en.y + en.z * en.z;
            const float sc = spiky_scale(P, r2);
            float f = li + en.w;
            if (P.scorr) {  // computeSCorr, CS_ComputeDeltaP.glsl:94-104
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
                    f -= P.k_corr * pw;
                }
            }
            const float g = sc * f;
            dx += en.x * g;
            dy += en.y * g;
            dz += en.z * g;
        });
    if (!active) return;
    dx *= P.inv_rho0;
    dy *= P.inv_rho0;
    dz *= P.inv_rho0;
    const float l2 = dx * dx + dy * dy + dz * dz;
    if (l2 > P.max_dp * P.max_dp) {
        const float sc = P.max_dp * rsqrtf(l2);
        dx *= sc;
        dy *= sc;
        dz *= sc;
    }
    float3 p = make_float3(xi.x + dx, xi.y + dy, xi.z + dz);
    if (P.sdf.enabled) {
        float3 nrm;
        sdf_project(P.sdf, p, nrm);
    }
    xout[s] = make_float4(p.x, p.y, p.z, li);
}

// ---- CS_Integrate.glsl:135-280 (pre-dispatch neighbour velocities) -------------------------------
__global__ void __launch_bounds__(kQThreads) k_integrate_q(DevParams P, const float4* __restrict__ xs,
                                                           const float4* __restrict__ sv, float4* __restrict__ sx0,
                                                           float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ pos,
                                                           float4* __restrict__ vel, const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order)
{
    __shared__ float4 rings[kQDepth * kQThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (order ? (int)__ldg(order + t) : t) : -1;
    float4 x4 = make_float4(0.f, 0.f, 0.f, 0.f), v0 = x4;
    if (in) {
        x4 = __ldg(xs + s);
        v0 = __ldg(sv + s);
    }
    float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    const bool walk = in && (P.visc_on || P.vort_on);
    queued_walk(
        P, table, walk, x4.x, x4.y, x4.z, s, rings + threadIdx.x,
        [&](int k, float4& ent) {
            const float4 xj = __ldg(xs + k);
            const float rx = x4.x - xj.x, ry = x4.y - xj.y, rz = x4.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            ent = make_float4(rx, ry, rz, __int_as_float(k));
            return r2 <= P.h2;
        },
        [&](const float4& en) {
            const float r2 = en.x * en.x + en.y * en.y + en.z * en.z;
            const float4 vj = __ldg(sv + __float_as_int(en.w));
            const float ux = vj.x - v0.x, uy = vj.y - v0.y, uz = vj.z - v0.z;
            if (P.visc_on) {
                const float w = poly6_in(P, r2) * P.inv_rho0;
                fx += ux * w;
                fy += uy * w;
                fz += uz * w;
            }
            if (P.vort_on && r2 >= 1e-10f) {
                const float sc = spiky_scale(P, r2);
                const float ax = en.x * sc, ay = en.y * sc, az = en.z * sc;
                cx += uy * az - uz * ay;
                cy += uz * ax - ux * az;
                cz += ux * ay - uy * ax;
            }
        });
    if (!in) return;
    const float4 p0 = sx0[s];
    float3 x = make_float3(x4.x, x4.y, x4.z);
    float vdx = 0.f, vdy = 0.f, vdz = 0.f;
    if (P.visc_on) {
        vdx = fx * P.viscosity;
        vdy = fy * P.viscosity;
        vdz = fz * P.viscosity;
    }
    if (P.vort_on) {
        const float ox = cx * P.inv_rho0, oy = cy * P.inv_rho0, oz = cz * P.inv_rho0;
        somega[s] = make_float4(ox, oy, oz, sqrtf(ox * ox + oy * oy + oz * oz));
    }
    bool colx = false, coly = false, colz = false;
    if (x.x <= P.bmin[0]) { x.x = P.bmin[0]; colx = true; }
    if (x.x >= P.bmax[0]) { x.x = P.bmax[0]; colx = true; }
    if (x.y <= P.bmin[1]) { x.y = P.bmin[1]; coly = true; }
    if (x.y >= P.bmax[1]) { x.y = P.bmax[1]; coly = true; }
    if (x.z <= P.bmin[2]) { x.z = P.bmin[2]; colz = true; }
    if (x.z >= P.bmax[2]) { x.z = P.bmax[2]; colz = true; }
    bool col_sdf = false;
    float3 nrm = make_float3(0.0f, 0.0f, 0.0f);
    if (P.sdf.enabled) col_sdf = sdf_project(P.sdf, x, nrm);
    float vx = (x.x - p0.x) * P.inv_dt + vdx;
    float vy = (x.y - p0.y) * P.inv_dt + vdy;
    float vz = (x.z - p0.z) * P.inv_dt + vdz;
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
    const uint32_t id = __ldg(ids + s);
    const float4 xo = make_float4(x.x, x.y, x.z, p0.w);
    pos[id] = xo;
    vel[id] = make_float4(vx, vy, vz, v0.w);
    sx0[s] = xo;
}

// ---- CS_VorticityConfinement.glsl:133-167 (pass 1) ------------------------------------------------
__global__ void __launch_bounds__(kQThreads) k_vorticity_q(DevParams P, const float4* __restrict__ spos,
                                                           const float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ vel,
                                                           const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order)
{
    __shared__ float4 rings[kQDepth * kQThreads];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (order ? (int)__ldg(order + t) : t) : -1;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in) xi = __ldg(spos + s);
    float ex = 0.f, ey = 0.f, ez = 0.f;
    queued_walk(
        P, table, in, xi.x, xi.y, xi.z, s, rings + threadIdx.x,
        [&](int k, float4& ent) {
            const float4 xj = __ldg(spos + k);
            const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            ent = make_float4(rx, ry, rz, __int_as_float(k));
            return r2 <= P.h2 && r2 >= 1e-10f;
        },
        [&](const float4& en) {
            const float r2 = en.x * en.x + en.y * en.y + en.z * en.z;
            const float sc = spiky_scale(P, r2) * __ldg(&somega[__float_as_int(en.w)].w);
            ex += en.x * sc;
            ey += en.y * sc;
            ez += en.z * sc;
        });
    if (!in) return;
    ex *= P.inv_rho0;
    ey *= P.inv_rho0;
    ez *= P.inv_rho0;
    const float el = sqrtf(ex * ex + ey * ey + ez * ez);
    if (el < 1e-6f) return;
    const float nx = ex / el, ny = ey / el, nz = ez / el;
    const float4 w = __ldg(somega + s);
    const float crx = ny * w.z - nz * w.y, cry = nz * w.x - nx * w.z, crz = nx * w.y - ny * w.x;
    const uint32_t id = __ldg(ids + s);
    float4 v = vel[id];
    v.x += P.vort_eps * crx * P.dt;
    v.y += P.vort_eps * cry * P.dt;
    v.z += P.vort_eps * crz * P.dt;
    vel[id] = v;
}

static inline unsigned qgrid(uint32_t n) { return (n + kQThreads - 1) / kQThreads; }

void launch_lambda_q(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                     const uint32_t* lod, uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    k_lambda_q<<<qgrid(P.n), kQThreads, 0, st>>>(P, xin, xout, rho, table, lod, iter, order);
}

void launch_deltap_q(const DevParams& P, const float4* xin, float4* xout, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    k_deltap_q<<<qgrid(P.n), kQThreads, 0, st>>>(P, xin, xout, table, lod, iter, order);
}

void launch_integrate_q(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                        const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                        cudaStream_t st)
{
    k_integrate_q<<<qgrid(P.n), kQThreads, 0, st>>>(P, xs, sv, sx0, somega, ids, pos, vel, table, order);
}

void launch_vorticity_q(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                        float4* vel, const int2* table, const uint32_t* order, cudaStream_t st)
{
    k_vorticity_q<<<qgrid(P.n), kQThreads, 0, st>>>(P, spos, somega, ids, vel, table, order);
}

}  // namespace pbf
