// k_solver.cu — the per-substep passes of the PBF solver on sm_100a.
//
// One thread per particle (particle order) or per sorted slot.  Neighbour
// passes read candidates from the sorted float4 arrays through the read-only
// path (__ldg), so a bucket's run of float4 is served from L1 once fetched by
// any thread of the block.
#include "pbf_kernels.h"

namespace pbf {

// CS_PredictAndHash.glsl:88-130 — only the key is stored; x* and v' are
// re-derived bit-identically by the reorder kernel after the sort.
__global__ void __launch_bounds__(256) k_predict_hash(DevParams P, const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel, uint32_t* __restrict__ keys)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        float3 vp, xs;
        predict_particle(P, __ldg(pos + i), __ldg(vel + i), vp, xs);
        keys[i] = grid_hash(cell_coord(xs.x, P.h), cell_coord(xs.y, P.h), cell_coord(xs.z, P.h), P.mask);
    }
}

// 8 low bits of a cell coordinate spread to every third bit.
__device__ __forceinline__ uint32_t spread8(uint32_t v)
{
    v &= 0xFFu;
    v = (v | (v << 8)) & 0x0000F00Fu;
    v = (v | (v << 4)) & 0x000C30C3u;
    v = (v | (v << 2)) & 0x00249249u;
    return v;
}

// Gather into sorted order: x* (lambda = 0, CS_PredictAndHash.glsl:121),
// v' and x, plus the APBF level of CS_ComputeLOD.glsl:66-79, and the 24-bit
// Morton code of the predict-time cell (low 8 bits per axis) that orders the
// neighbour passes' threads spatially.
__global__ void __launch_bounds__(256) k_reorder(DevParams P, const uint32_t* __restrict__ ids,
                                                 const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                 float4* __restrict__ sx, float4* __restrict__ sv,
                                                 float4* __restrict__ sx0, uint32_t* __restrict__ lod,
                                                 uint32_t* __restrict__ mcode)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.n; s += stride) {
        const uint32_t id = __ldg(ids + s);
        const float4 p = __ldg(pos + id);
        const float4 v = __ldg(vel + id);
        float3 vp, xs;
        predict_particle(P, p, v, vp, xs);
        sx[s] = make_float4(xs.x, xs.y, xs.z, 0.0f);
        sv[s] = make_float4(vp.x, vp.y, vp.z, v.w);
        sx0[s] = p;
        if (mcode) {
            const uint32_t cx = (uint32_t)cell_coord(xs.x, P.h), cy = (uint32_t)cell_coord(xs.y, P.h),
                           cz = (uint32_t)cell_coord(xs.z, P.h);
            mcode[s] = (spread8(cz) << 2) | (spread8(cy) << 1) | spread8(cx);
        }
        if (P.apbf) {
            const float dx = P.cam[0] - xs.x, dy = P.cam[1] - xs.y, dz = P.cam[2] - xs.z;
            const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
            const float t = fminf(fmaxf(dist / P.lod_max_dist, 0.0f), 1.0f);
            const float m = (float)P.max_lod * (1.0f - t) + (float)P.min_lod * t;
            uint32_t l = (uint32_t)rintf(m);
            l = min(max(l, P.min_lod), P.max_lod);
            lod[s] = l;
        }
    }
}

// CS_BuildOffsets.glsl:63-78 (the clear is a memset of 0xFF = -1).
__global__ void __launch_bounds__(256) k_build_table(uint32_t n, const uint32_t* __restrict__ sk,
                                                     int2* __restrict__ table)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t k = __ldg(sk + i);
        if (i == 0 || __ldg(sk + i - 1) != k) table[k].x = (int)i;
        if (i == n - 1 || __ldg(sk + i + 1) != k) table[k].y = (int)(i + 1);
    }
}

// CS_ComputeLambdas.glsl:108-162.  Reads (x*, .) from xin, writes (x*, lambda)
// to xout; inactive APBF particles carry their previous lambda.
__global__ void __launch_bounds__(128) k_lambda(DevParams P, const float4* __restrict__ xin,
                                                float4* __restrict__ xout, float* __restrict__ rho_out,
                                                const int2* __restrict__ table, const uint32_t* __restrict__ lod,
                                                uint32_t iter, const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    const float4 xi = __ldg(xin + s);
    if (P.apbf && __ldg(lod + s) < iter) {
        xout[s] = xi;
        return;
    }
    float rho = P.w0_self;
    float sg = 0.0f;
    float gx = 0.0f, gy = 0.0f, gz = 0.0f;
    for_each_neighbour(P, table, xi.x, xi.y, xi.z, s, [&](int k) {
        const float4 xj = __ldg(xin + k);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        if (r2 <= P.h2) {
            rho += poly6_in(P, r2);
            if (r2 >= 1e-10f) {
                const float sc = spiky_scale(P, r2);
                const float ax = rx * sc, ay = ry * sc, az = rz * sc;
                sg += (ax * ax + ay * ay + az * az) * P.inv_rho0_sq;
                gx += ax;
                gy += ay;
                gz += az;
            }
        }
    });
    gx *= P.inv_rho0;
    gy *= P.inv_rho0;
    gz *= P.inv_rho0;
    const float C = fmaxf(rho / P.rho0 - 1.0f, -P.cohesion);
    sg += gx * gx + gy * gy + gz * gz;
    const float lambda = -C / (sg + P.eps);
    xout[s] = make_float4(xi.x, xi.y, xi.z, lambda);
    rho_out[s] = rho;
}

// CS_ComputeDeltaP.glsl:120-166 fused with CS_ApplyDeltaP.glsl:80-124.  The
// two reference dispatches are separated only so that every dp reads the same
// x*; here that is guaranteed by reading xin and writing xout (Jacobi).
__global__ void __launch_bounds__(128) k_deltap_apply(DevParams P, const float4* __restrict__ xin,
                                                      float4* __restrict__ xout, const int2* __restrict__ table,
                                                      const uint32_t* __restrict__ lod, uint32_t iter,
                                                      const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    const float4 xi = __ldg(xin + s);
    if (P.apbf && __ldg(lod + s) < iter) {
        xout[s] = xi;
        return;
    }
    const float li = xi.w;
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    for_each_neighbour(P, table, xi.x, xi.y, xi.z, s, [&](int k) {
        const float4 xj = __ldg(xin + k);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        if (r2 <= P.h2 && r2 >= 1e-10f) {
            const float sc = spiky_scale(P, r2);
            const float f = li + xj.w + (r2 < P.h2 ? scorr_in(P, r2) : 0.0f);
            dx += rx * sc * f;
            dy += ry * sc * f;
            dz += rz * sc * f;
        }
    });
    dx *= P.inv_rho0;
    dy *= P.inv_rho0;
    dz *= P.inv_rho0;
    const float l2 = dx * dx + dy * dy + dz * dz;
    if (l2 > P.max_dp * P.max_dp) {
        const float sc = P.max_dp / sqrtf(l2);
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

// CS_Integrate.glsl:135-280 with pre-dispatch neighbour velocities (sv is
// never written here).  Commits x and v to particle order, keeps the
// committed x in sorted order (sx0, in place) and omega for vorticity.
__global__ void __launch_bounds__(128) k_integrate(DevParams P, const float4* __restrict__ xs,
                                                   const float4* __restrict__ sv, float4* __restrict__ sx0,
                                                   float4* __restrict__ somega, const uint32_t* __restrict__ ids,
                                                   float4* __restrict__ pos, float4* __restrict__ vel,
                                                   const int2* __restrict__ table, const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    const float4 x4 = __ldg(xs + s);
    const float4 v0 = __ldg(sv + s);
    const float4 p0 = sx0[s];
    float3 x = make_float3(x4.x, x4.y, x4.z);
    float vdx = 0.0f, vdy = 0.0f, vdz = 0.0f;
    if (P.visc_on || P.vort_on) {
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        float cx = 0.0f, cy = 0.0f, cz = 0.0f;
        for_each_neighbour(P, table, x.x, x.y, x.z, s, [&](int k) {
            const float4 xj = __ldg(xs + k);
            const float rx = x.x - xj.x, ry = x.y - xj.y, rz = x.z - xj.z;
            const float r2 = rx * rx + ry * ry + rz * rz;
            if (r2 <= P.h2) {
                const float4 vj = __ldg(sv + k);
                const float ux = vj.x - v0.x, uy = vj.y - v0.y, uz = vj.z - v0.z;
                if (P.visc_on) {
                    const float w = poly6_in(P, r2);
                    fx += ux * w * P.inv_rho0;
                    fy += uy * w * P.inv_rho0;
                    fz += uz * w * P.inv_rho0;
                }
                if (P.vort_on && r2 >= 1e-10f) {
                    const float sc = spiky_scale(P, r2);
                    const float ax = rx * sc, ay = ry * sc, az = rz * sc;
                    cx += uy * az - uz * ay;
                    cy += uz * ax - ux * az;
                    cz += ux * ay - uy * ax;
                }
            }
        });
        if (P.visc_on) {
            vdx = fx * P.viscosity;
            vdy = fy * P.viscosity;
            vdz = fz * P.viscosity;
        }
        if (P.vort_on) {
            const float ox = cx * P.inv_rho0, oy = cy * P.inv_rho0, oz = cz * P.inv_rho0;
            somega[s] = make_float4(ox, oy, oz, sqrtf(ox * ox + oy * oy + oz * oz));
        }
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

// CS_VorticityConfinement.glsl:133-167 (pass 1) over the last substep's
// buckets, committed positions and omega.
__global__ void __launch_bounds__(128) k_vorticity(DevParams P, const float4* __restrict__ spos,
                                                   const float4* __restrict__ somega,
                                                   const uint32_t* __restrict__ ids, float4* __restrict__ vel,
                                                   const int2* __restrict__ table, const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    const float4 xi = __ldg(spos + s);
    float ex = 0.0f, ey = 0.0f, ez = 0.0f;
    for_each_neighbour(P, table, xi.x, xi.y, xi.z, s, [&](int k) {
        const float4 xj = __ldg(spos + k);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        const float r2 = rx * rx + ry * ry + rz * rz;
        if (r2 <= P.h2 && r2 >= 1e-10f) {
            const float sc = spiky_scale(P, r2) * __ldg(&somega[k].w);
            ex += rx * sc;
            ey += ry * sc;
            ez += rz * sc;
        }
    });
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

__global__ void k_check_finite(uint32_t n, const float4* __restrict__ pos, const float4* __restrict__ vel,
                               uint32_t* __restrict__ bad)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    uint32_t c = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float4 p = pos[i], v = vel[i];
        if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z) || !isfinite(v.x) || !isfinite(v.y) ||
            !isfinite(v.z))
            ++c;
    }
    if (c) atomicAdd(bad, c);
}

// Particle {vec4 pos, predPos, vel} (Particle.h:8-12) <-> engine arrays.
__global__ void k_unpack_particles(uint32_t n, const float4* __restrict__ aos, float4* __restrict__ pos,
                                   float4* __restrict__ pred, float4* __restrict__ vel)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        pos[i] = __ldg(aos + 3 * (size_t)i);
        pred[i] = __ldg(aos + 3 * (size_t)i + 1);
        vel[i] = __ldg(aos + 3 * (size_t)i + 2);
    }
}

__global__ void k_pack_particles(uint32_t n, const float4* __restrict__ pos, const float4* __restrict__ pred,
                                 const float4* __restrict__ vel, float4* __restrict__ aos)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        aos[3 * (size_t)i] = __ldg(pos + i);
        aos[3 * (size_t)i + 1] = __ldg(pred + i);
        aos[3 * (size_t)i + 2] = __ldg(vel + i);
    }
}

// ---- launchers ---------------------------------------------------------------
static inline unsigned stream_grid(uint32_t n, int threads, int sms)
{
    const uint32_t want = (n + threads - 1) / threads;
    const uint32_t cap = (uint32_t)sms * 8u;
    return want < 1 ? 1 : (want > cap ? cap : want);
}

void launch_predict_hash(const DevParams& P, const float4* pos, const float4* vel, uint32_t* keys, int sms,
                         cudaStream_t st)
{
    k_predict_hash<<<stream_grid(P.n, 256, sms), 256, 0, st>>>(P, pos, vel, keys);
}

void launch_reorder(const DevParams& P, const uint32_t* ids, const float4* pos, const float4* vel, float4* sx,
                    float4* sv, float4* sx0, uint32_t* lod, uint32_t* mcode, int sms, cudaStream_t st)
{
    k_reorder<<<stream_grid(P.n, 256, sms), 256, 0, st>>>(P, ids, pos, vel, sx, sv, sx0, lod, mcode);
}

void launch_build_table(uint32_t n, const uint32_t* sk, int2* table, int sms, cudaStream_t st)
{
    k_build_table<<<stream_grid(n, 256, sms), 256, 0, st>>>(n, sk, table);
}

void launch_lambda(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                   const uint32_t* lod, uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    k_lambda<<<(P.n + 127) / 128, 128, 0, st>>>(P, xin, xout, rho, table, lod, iter, order);
}

void launch_deltap_apply(const DevParams& P, const float4* xin, float4* xout, const int2* table,
                         const uint32_t* lod, uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    k_deltap_apply<<<(P.n + 127) / 128, 128, 0, st>>>(P, xin, xout, table, lod, iter, order);
}

void launch_integrate(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                      const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                      cudaStream_t st)
{
    k_integrate<<<(P.n + 127) / 128, 128, 0, st>>>(P, xs, sv, sx0, somega, ids, pos, vel, table, order);
}

void launch_vorticity(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                      float4* vel, const int2* table, const uint32_t* order, cudaStream_t st)
{
    k_vorticity<<<(P.n + 127) / 128, 128, 0, st>>>(P, spos, somega, ids, vel, table, order);
}

void launch_check_finite(uint32_t n, const float4* pos, const float4* vel, uint32_t* bad, int sms,
                         cudaStream_t st)
{
    k_check_finite<<<stream_grid(n, 256, sms), 256, 0, st>>>(n, pos, vel, bad);
}

void launch_unpack_particles(uint32_t n, const float4* aos, float4* pos, float4* pred, float4* vel, int sms,
                             cudaStream_t st)
{
    k_unpack_particles<<<stream_grid(n, 256, sms), 256, 0, st>>>(n, aos, pos, pred, vel);
}

void launch_pack_particles(uint32_t n, const float4* pos, const float4* pred, const float4* vel, float4* aos,
                           int sms, cudaStream_t st)
{
    k_pack_particles<<<stream_grid(n, 256, sms), 256, 0, st>>>(n, pos, pred, vel, aos);
}

}  // namespace pbf
