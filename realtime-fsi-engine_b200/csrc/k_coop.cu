// k_coop.cu — cell-cooperative neighbour passes.
//
// The particles of one cell (one run of equal Morton codes in the spatial
// processing order, i.e. the members of one hash bucket that share a cell)
// are taken by one warp.  With c particles in the run, L = 8, 4, 2 or 1 lanes
// serve each particle (L*c <= 32) and stride through its candidate list, so
// the lanes of a warp walk the same 27 buckets in lock-step: every candidate
// load is a broadcast of one 16-byte float4 per stride position (one L1
// wavefront) and the loop trip counts agree across the warp.  The L partial
// sums of a particle are combined with a butterfly of shuffles.
//
// Each particle still walks the 27 buckets of its own current cell, so a
// particle that left the run's cell during the Jacobi iterations (or shares a
// bucket through a hash collision) gets its exact reference neighbour set;
// it only loses the broadcast.
#include "pbf_kernels.h"

namespace pbf {

constexpr int kCoopThreads = 128;

// Cell runs: starts of runs of equal codes in the sorted Morton list.
constexpr int kHeadItems = 8;
constexpr int kHeadBlock = 256 * kHeadItems;

__global__ void __launch_bounds__(256) k_head_count(uint32_t n, const uint32_t* __restrict__ codes,
                                                    uint32_t* __restrict__ counts)
{
    uint32_t c = 0;
    const uint32_t base = blockIdx.x * kHeadBlock;
#pragma unroll
    for (int r = 0; r < kHeadItems; ++r) {
        const uint32_t i = base + r * 256 + threadIdx.x;
        if (i < n && (i == 0 || __ldg(codes + i) != __ldg(codes + i - 1))) ++c;
    }
    __shared__ uint32_t sm[8];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < 8; ++w) t += sm[w];
        counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(1024) k_head_scan(uint32_t* __restrict__ counts, uint32_t nb,
                                                    uint32_t* __restrict__ total)
{
    __shared__ uint32_t ws[32];
    uint32_t carry = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nb; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nb ? counts[i] : 0u;
        uint32_t incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) ws[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = ws[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            ws[lane] = w;
        }
        __syncthreads();
        if (i < nb) counts[i] = carry + incl - v + (warp ? ws[warp - 1] : 0u);
        const uint32_t chunk = ws[31];
        __syncthreads();
        carry += chunk;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(256) k_head_write(uint32_t n, const uint32_t* __restrict__ codes,
                                                    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ total,
                                                    uint32_t* __restrict__ heads)
{
    __shared__ uint32_t ws[8];
    const uint32_t base = blockIdx.x * kHeadBlock;
    uint32_t run = offsets[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = 0; r < kHeadItems; ++r) {
        const uint32_t i = base + r * 256 + threadIdx.x;
        const bool f = i < n && (i == 0 || __ldg(codes + i) != __ldg(codes + i - 1));
        const uint32_t bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) ws[warp] = __popc(bal);
        __syncthreads();
        uint32_t woff = 0, all = 0;
        for (int w = 0; w < 8; ++w) {
            if (w < warp) woff += ws[w];
            all += ws[w];
        }
        if (f) heads[run + woff + __popc(bal & ((1u << lane) - 1u))] = i;
        run += all;
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) heads[*total] = n;  // sentinel end of the last run
}

uint32_t head_num_blocks(uint32_t n) { return (n + kHeadBlock - 1) / kHeadBlock; }

void launch_cell_runs(uint32_t n, const uint32_t* sorted_codes, uint32_t* block_counts, uint32_t* run_count,
                      uint32_t* run_starts, cudaStream_t st, uint64_t* launches)
{
    const uint32_t nb = head_num_blocks(n);
    k_head_count<<<nb, 256, 0, st>>>(n, sorted_codes, block_counts);
    k_head_scan<<<1, 1024, 0, st>>>(block_counts, nb, run_count);
    k_head_write<<<nb, 256, 0, st>>>(n, sorted_codes, block_counts, run_count, run_starts);
    if (launches) *launches += 3;
}

// ---- lane mapping ----------------------------------------------------------------------
struct Lane {
    int s;      // sorted slot of this lane's particle, -1 when the lane is idle
    int sub;    // index of this lane among its particle's L lanes
    int L;      // lanes per particle (uniform over the warp)
};

// Calls body(Lane) for every chunk of every cell run owned by this warp;
// every lane of the warp calls it (idle lanes with s = -1) so bodies may use
// full-warp shuffles.
template <class Body>
__device__ __forceinline__ void for_each_run(const uint32_t* __restrict__ order, const uint32_t* __restrict__ runs,
                                             const uint32_t* __restrict__ run_count, Body&& body)
{
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t G = __ldg(run_count);
    for (uint32_t g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; g < G; g += nwarps) {
        const uint32_t a = __ldg(runs + g), b = __ldg(runs + g + 1);
        for (uint32_t c0 = a; c0 < b; c0 += 32) {
            const uint32_t c = min(b - c0, 32u);
            const int L = c <= 4 ? 8 : (c <= 8 ? 4 : (c <= 16 ? 2 : 1));
            const int shift = L == 8 ? 3 : (L == 4 ? 2 : (L == 2 ? 1 : 0));
            Lane ln;
            const uint32_t pi = (uint32_t)lane >> shift;
            ln.sub = lane & (L - 1);
            ln.L = L;
            ln.s = pi < c ? (int)__ldg(order + c0 + pi) : -1;
            body(ln);
        }
    }
}

__device__ __forceinline__ float lane_sum(float v, int L)
{
    for (int o = 1; o < L; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Strided walk of the 27 buckets of the particle's current cell.
template <class Fn>
__device__ __forceinline__ void walk(const DevParams& P, const int2* __restrict__ table, float xi, float yi, float zi,
                                     int self, int sub, int L, Fn&& fn)
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
                for (int k = se.x + sub; k < se.y; k += L) {
                    if (k == self) continue;
                    fn(k);
                }
            }
        }
    }
}

__device__ __forceinline__ float spiky_fast(const DevParams& P, float r2) { return spiky_scale(P, r2); }

// ---- CS_ComputeLambdas.glsl:108-162 -----------------------------------------------------
__global__ void __launch_bounds__(kCoopThreads) k_lambda_coop(DevParams P, const float4* __restrict__ xin,
                                                              float4* __restrict__ xout, float* __restrict__ rho_out,
                                                              const int2* __restrict__ table,
                                                              const uint32_t* __restrict__ lod, uint32_t iter,
                                                              const uint32_t* __restrict__ order,
                                                              const uint32_t* __restrict__ runs,
                                                              const uint32_t* __restrict__ run_count)
{
    for_each_run(order, runs, run_count, [&](const Lane& ln) {
        float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
        bool act = ln.s >= 0;
        if (act) {
            xi = __ldg(xin + ln.s);
            if (P.apbf && __ldg(lod + ln.s) < iter) {
                if (ln.sub == 0) xout[ln.s] = xi;
                act = false;
            }
        }
        float rho = 0.f, sg = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
        if (act) {
            walk(P, table, xi.x, xi.y, xi.z, ln.s, ln.sub, ln.L, [&](int k) {
                const float4 xj = __ldg(xin + k);
                const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (r2 <= P.h2) {
                    rho += poly6_in(P, r2);
                    if (r2 >= 1e-10f) {
                        const float sc = spiky_fast(P, r2);
                        const float ax = rx * sc, ay = ry * sc, az = rz * sc;
                        sg += (ax * ax + ay * ay + az * az) * P.inv_rho0_sq;
                        gx += ax;
                        gy += ay;
                        gz += az;
                    }
                }
            });
        }
        rho = lane_sum(rho, ln.L);
        sg = lane_sum(sg, ln.L);
        gx = lane_sum(gx, ln.L);
        gy = lane_sum(gy, ln.L);
        gz = lane_sum(gz, ln.L);
        if (act && ln.sub == 0) {
            rho += P.w0_self;
            gx *= P.inv_rho0;
            gy *= P.inv_rho0;
            gz *= P.inv_rho0;
            const float C = fmaxf(rho / P.rho0 - 1.0f, -P.cohesion);
            sg += gx * gx + gy * gy + gz * gz;
            xout[ln.s] = make_float4(xi.x, xi.y, xi.z, -C / (sg + P.eps));
            rho_out[ln.s] = rho;
        }
    });
}

// ---- CS_ComputeDeltaP.glsl:120-166 + CS_ApplyDeltaP.glsl:80-124 ------------------------------
__global__ void __launch_bounds__(kCoopThreads) k_deltap_coop(DevParams P, const float4* __restrict__ xin,
                                                              float4* __restrict__ xout, const int2* __restrict__ table,
                                                              const uint32_t* __restrict__ lod, uint32_t iter,
                                                              const uint32_t* __restrict__ order,
                                                              const uint32_t* __restrict__ runs,
                                                              const uint32_t* __restrict__ run_count)
{
    for_each_run(order, runs, run_count, [&](const Lane& ln) {
        float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
        bool act = ln.s >= 0;
        if (act) {
            xi = __ldg(xin + ln.s);
            if (P.apbf && __ldg(lod + ln.s) < iter) {
                if (ln.sub == 0) xout[ln.s] = xi;
                act = false;
            }
        }
        float dx = 0.f, dy = 0.f, dz = 0.f;
        if (act) {
            const float li = xi.w;
            walk(P, table, xi.x, xi.y, xi.z, ln.s, ln.sub, ln.L, [&](int k) {
                const float4 xj = __ldg(xin + k);
                const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (r2 <= P.h2 && r2 >= 1e-10f) {
                    const float sc = spiky_fast(P, r2);
                    float f = li + xj.w;
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
                    dx += rx * g;
                    dy += ry * g;
                    dz += rz * g;
                }
            });
        }
        dx = lane_sum(dx, ln.L);
        dy = lane_sum(dy, ln.L);
        dz = lane_sum(dz, ln.L);
        if (act && ln.sub == 0) {
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
            xout[ln.s] = make_float4(p.x, p.y, p.z, xi.w);
        }
    });
}

// ---- CS_Integrate.glsl:135-280 (pre-dispatch neighbour velocities) -------------------------------
__global__ void __launch_bounds__(kCoopThreads) k_integrate_coop(DevParams P, const float4* __restrict__ xs,
                                                                 const float4* __restrict__ sv, float4* __restrict__ sx0,
                                                                 float4* __restrict__ somega,
                                                                 const uint32_t* __restrict__ ids,
                                                                 float4* __restrict__ pos, float4* __restrict__ vel,
                                                                 const int2* __restrict__ table,
                                                                 const uint32_t* __restrict__ order,
                                                                 const uint32_t* __restrict__ runs,
                                                                 const uint32_t* __restrict__ run_count)
{
    for_each_run(order, runs, run_count, [&](const Lane& ln) {
        const bool act = ln.s >= 0;
        float4 x4 = make_float4(0.f, 0.f, 0.f, 0.f), v0 = x4;
        if (act) {
            x4 = __ldg(xs + ln.s);
            v0 = __ldg(sv + ln.s);
        }
        float fx = 0.f, fy = 0.f, fz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
        if (act && (P.visc_on || P.vort_on)) {
            walk(P, table, x4.x, x4.y, x4.z, ln.s, ln.sub, ln.L, [&](int k) {
                const float4 xj = __ldg(xs + k);
                const float rx = x4.x - xj.x, ry = x4.y - xj.y, rz = x4.z - xj.z;
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (r2 <= P.h2) {
                    const float4 vj = __ldg(sv + k);
                    const float ux = vj.x - v0.x, uy = vj.y - v0.y, uz = vj.z - v0.z;
                    if (P.visc_on) {
                        const float w = poly6_in(P, r2) * P.inv_rho0;
                        fx += ux * w;
                        fy += uy * w;
                        fz += uz * w;
                    }
                    if (P.vort_on && r2 >= 1e-10f) {
                        const float sc = spiky_fast(P, r2);
                        const float ax = rx * sc, ay = ry * sc, az = rz * sc;
                        cx += uy * az - uz * ay;
                        cy += uz * ax - ux * az;
                        cz += ux * ay - uy * ax;
                    }
                }
            });
        }
        fx = lane_sum(fx, ln.L);
        fy = lane_sum(fy, ln.L);
        fz = lane_sum(fz, ln.L);
        cx = lane_sum(cx, ln.L);
        cy = lane_sum(cy, ln.L);
        cz = lane_sum(cz, ln.L);
        if (!act || ln.sub != 0) return;
        const float4 p0 = sx0[ln.s];
        float3 x = make_float3(x4.x, x4.y, x4.z);
        float vdx = 0.f, vdy = 0.f, vdz = 0.f;
        if (P.visc_on) {
            vdx = fx * P.viscosity;
            vdy = fy * P.viscosity;
            vdz = fz * P.viscosity;
        }
        if (P.vort_on) {
            const float ox = cx * P.inv_rho0, oy = cy * P.inv_rho0, oz = cz * P.inv_rho0;
            somega[ln.s] = make_float4(ox, oy, oz, sqrtf(ox * ox + oy * oy + oz * oz));
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
        const uint32_t id = __ldg(ids + ln.s);
        const float4 xo = make_float4(x.x, x.y, x.z, p0.w);
        pos[id] = xo;
        vel[id] = make_float4(vx, vy, vz, v0.w);
        sx0[ln.s] = xo;
    });
}

// ---- CS_VorticityConfinement.glsl:133-167 (pass 1) ------------------------------------------------
__global__ void __launch_bounds__(kCoopThreads) k_vorticity_coop(DevParams P, const float4* __restrict__ spos,
                                                                 const float4* __restrict__ somega,
                                                                 const uint32_t* __restrict__ ids,
                                                                 float4* __restrict__ vel,
                                                                 const int2* __restrict__ table,
                                                                 const uint32_t* __restrict__ order,
                                                                 const uint32_t* __restrict__ runs,
                                                                 const uint32_t* __restrict__ run_count)
{
    for_each_run(order, runs, run_count, [&](const Lane& ln) {
        const bool act = ln.s >= 0;
        float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
        if (act) xi = __ldg(spos + ln.s);
        float ex = 0.f, ey = 0.f, ez = 0.f;
        if (act) {
            walk(P, table, xi.x, xi.y, xi.z, ln.s, ln.sub, ln.L, [&](int k) {
                const float4 xj = __ldg(spos + k);
                const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (r2 <= P.h2 && r2 >= 1e-10f) {
                    const float sc = spiky_fast(P, r2) * __ldg(&somega[k].w);
                    ex += rx * sc;
                    ey += ry * sc;
                    ez += rz * sc;
                }
            });
        }
        ex = lane_sum(ex, ln.L);
        ey = lane_sum(ey, ln.L);
        ez = lane_sum(ez, ln.L);
        if (!act || ln.sub != 0) return;
        ex *= P.inv_rho0;
        ey *= P.inv_rho0;
        ez *= P.inv_rho0;
        const float el = sqrtf(ex * ex + ey * ey + ez * ez);
        if (el < 1e-6f) return;
        const float nx = ex / el, ny = ey / el, nz = ez / el;
        const float4 w = __ldg(somega + ln.s);
        const float crx = ny * w.z - nz * w.y, cry = nz * w.x - nx * w.z, crz = nx * w.y - ny * w.x;
        const uint32_t id = __ldg(ids + ln.s);
        float4 v = vel[id];
        v.x += P.vort_eps * crx * P.dt;
        v.y += P.vort_eps * cry * P.dt;
        v.z += P.vort_eps * crz * P.dt;
        vel[id] = v;
    });
}

static inline unsigned coop_grid(int sms) { return (unsigned)sms * 16u; }

void launch_lambda_coop(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                        const uint32_t* lod, uint32_t iter, const uint32_t* order, const uint32_t* runs,
                        const uint32_t* run_count, int sms, cudaStream_t st)
{
    k_lambda_coop<<<coop_grid(sms), kCoopThreads, 0, st>>>(P, xin, xout, rho, table, lod, iter, order, runs,
                                                           run_count);
}

void launch_deltap_coop(const DevParams& P, const float4* xin, float4* xout, const int2* table, const uint32_t* lod,
                        uint32_t iter, const uint32_t* order, const uint32_t* runs, const uint32_t* run_count, int sms,
                        cudaStream_t st)
{
    k_deltap_coop<<<coop_grid(sms), kCoopThreads, 0, st>>>(P, xin, xout, table, lod, iter, order, runs, run_count);
}

void launch_integrate_coop(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                           const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                           const uint32_t* runs, const uint32_t* run_count, int sms, cudaStream_t st)
{
    k_integrate_coop<<<coop_grid(sms), kCoopThreads, 0, st>>>(P, xs, sv, sx0, somega, ids, pos, vel, table, order,
                                                              runs, run_count);
}

void launch_vorticity_coop(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                           float4* vel, const int2* table, const uint32_t* order, const uint32_t* runs,
                           const uint32_t* run_count, int sms, cudaStream_t st)
{
    k_vorticity_coop<<<coop_grid(sms), kCoopThreads, 0, st>>>(P, spos, somega, ids, vel, table, order, runs,
                                                              run_count);
}

}  // namespace pbf
