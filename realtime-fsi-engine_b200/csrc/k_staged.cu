// k_staged.cu — neighbour passes staged through shared memory per cell block.
//
// A block takes 256 particles that are consecutive in the Morton order of
// their cells — a compact block of ~32 cells.  Its threads' 27-bucket
// neighbourhoods overlap heavily, so the block:
//   1. inserts the hash of every bucket any of its threads will walk into a
//      shared-memory hash set (open addressing, atomicCAS);
//   2. reads the (start, end) table entry of each distinct bucket and lays
//      the buckets out back to back (block-wide scan of their sizes);
//   3. copies the candidates of every distinct bucket into shared memory with
//      one coalesced warp load per bucket;
//   4. lets every thread walk its own 27 buckets out of shared memory, with
//      the per-bucket hit mask of k_masked.cu (chunks of 8 tested first, the
//      pair body run only for the hits).
// Each candidate is fetched from L2/HBM once per block instead of once per
// thread that visits it.  A block whose distinct buckets hold more
// candidates than fit falls back to reading them from global memory.  Either
// way every particle visits exactly its reference candidate multiset in the
// reference's order.
#include "pbf_kernels.h"

namespace pbf {

constexpr int kSThreads = 256;
constexpr int kHashSlots = 1024;  // shared hash set of bucket ids (power of two)
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

struct StagedShared {
    uint32_t key[kHashSlots];    // bucket hash or kEmpty
    int start[kHashSlots];       // global slot of the bucket's first candidate
    int count[kHashSlots];       // bucket size
    int off[kHashSlots];         // offset of the bucket in the staged arrays
    int warp_tot[kSThreads / 32];
    int total;
    int overflow;
};

// Both probes visit each slot at most once, so they end even on a full set.
__device__ __forceinline__ int hs_probe(const uint32_t* key, uint32_t h)
{
    uint32_t i = (h * 2654435761u) & (kHashSlots - 1);
    for (int n = 0; n < kHashSlots; ++n) {
        const uint32_t k = key[i];
        if (k == h) return (int)i;
        if (k == kEmpty) return -1;
        i = (i + 1) & (kHashSlots - 1);
    }
    return -1;
}

__device__ __forceinline__ bool hs_insert(uint32_t* key, uint32_t h)
{
    uint32_t i = (h * 2654435761u) & (kHashSlots - 1);
    for (int n = 0; n < kHashSlots; ++n) {
        const uint32_t prev = atomicCAS(key + i, kEmpty, h);
        if (prev == kEmpty || prev == h) return true;
        i = (i + 1) & (kHashSlots - 1);
    }
    return false;
}

// Bucket hash of neighbour b (0..26, z outer / x inner) of a cell.
__device__ __forceinline__ uint32_t nb_hash(const DevParams& P, int cx, int cy, int cz, int b)
{
    return grid_hash(cx + b % 3 - 1, cy + (b / 3) % 3 - 1, cz + b / 9 - 1, P.mask);
}

// Stages the candidate data of all buckets walked by the block's particles.
// `stage(k, dst_index)` copies candidate slot k into the staged arrays.
// Returns false when the block must read candidates from global memory.
template <class Stage>
__device__ bool stage_block(const DevParams& P, const int2* __restrict__ table, StagedShared& S, bool have, int cx,
                            int cy, int cz, int cap, Stage&& stage)
{
    for (int i = threadIdx.x; i < kHashSlots; i += kSThreads) S.key[i] = kEmpty;
    if (threadIdx.x == 0) S.overflow = 0;
    __syncthreads();
    // Threads come in Morton order, so a cell's particles are neighbours in
    // the block: only the first thread of each run of equal cells inserts
    // (the others would CAS the same 27 words and serialise on them).
    {
        const int pcx = __shfl_up_sync(0xffffffffu, cx, 1), pcy = __shfl_up_sync(0xffffffffu, cy, 1),
                  pcz = __shfl_up_sync(0xffffffffu, cz, 1);
        const bool phave = __shfl_up_sync(0xffffffffu, (int)have, 1) != 0;
        const bool first = (threadIdx.x & 31) == 0 || !phave || pcx != cx || pcy != cy || pcz != cz;
        if (have && first) {
            bool ok = true;
            for (int b = 0; b < 27; ++b) ok &= hs_insert(S.key, nb_hash(P, cx, cy, cz, b));
            if (!ok) atomicOr(&S.overflow, 1);  // too many distinct buckets: read from global memory
        }
    }
    __syncthreads();
    // sizes of the distinct buckets, laid out by a block-wide exclusive scan
    constexpr int kPer = kHashSlots / kSThreads;
    int cnt[kPer];
    int local = 0;
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        const int i = threadIdx.x * kPer + r;
        cnt[r] = 0;
        const uint32_t k = S.key[i];
        if (k != kEmpty) {
            const int2 se = __ldg(table + k);
            if (se.x != -1) {
                cnt[r] = se.y - se.x;
                S.start[i] = se.x;
            }
        }
        S.count[i] = cnt[r];
        local += cnt[r];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) S.warp_tot[warp] = incl;
    __syncthreads();
    int base = 0, all = 0;
#pragma unroll
    for (int w = 0; w < kSThreads / 32; ++w) {
        if (w < warp) base += S.warp_tot[w];
        all += S.warp_tot[w];
    }
    int run = base + incl - local;
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        S.off[threadIdx.x * kPer + r] = run;
        run += cnt[r];
    }
    if (threadIdx.x == 0) {
        S.total = all;
        if (all > cap) S.overflow = 1;
    }
    __syncthreads();
    if (S.overflow) return false;
    // copy: warp w copies the buckets in hash slots w, w+8, ...; lane = entry
    for (int i = warp; i < kHashSlots; i += kSThreads / 32) {
        const int c = S.count[i];
        if (c == 0) continue;
        const int g = S.start[i], o = S.off[i];
        for (int e = lane; e < c; e += 32) stage(g + e, o + e);
    }
    __syncthreads();
    return true;
}

// The particle's 27-bucket walk over staged candidates (or global memory
// after an overflow), testing chunks of 8 into a hit mask before the body.
// `pos(local_index)` returns the candidate float4 whose xyz is tested;
// body(local_index, global_slot) consumes one hit.
// One bucket: candidates [g, g+c) read through `get` (shared or global),
// tested in chunks of 8, hits passed to body(index for get, global slot).
template <class Get, class Hit, class Body>
__device__ __forceinline__ void bucket_hits(float xi, float yi, float zi, int self, int g, int c, int base, Get&& get,
                                            Hit&& hit, Body&& body)
{
#pragma unroll 1
    for (int e0 = 0; e0 < c; e0 += 8) {
        uint32_t m = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int e = e0 + u;
            if (e < c) {
                const float4 xj = get(base + e);
                const float rx = xi - xj.x, ry = yi - xj.y, rz = zi - xj.z;
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (hit(r2) && g + e != self) m |= 1u << u;
            }
        }
        while (m) {
            const int u = __ffs(m) - 1;
            m &= m - 1u;
            body(base + u + e0, g + u + e0);
        }
    }
}

// The particle's 27-bucket walk (z outer, x inner) over the staged
// candidates, or over global memory for a block that overflowed.
// loc(i) / glob(k) return a candidate from shared / global memory;
// body(is_local, index, global_slot) consumes one hit.
template <class Loc, class Glob, class Hit, class Body>
__device__ __forceinline__ void staged_walk(const DevParams& P, const int2* __restrict__ table, const StagedShared& S,
                                            bool staged, float xi, float yi, float zi, int cx, int cy, int cz, int self,
                                            Loc&& loc, Glob&& glob, Hit&& hit, Body&& body)
{
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
        const uint32_t hz = (uint32_t)(cz + dz) * kP3;
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
            const uint32_t hyz = hz ^ ((uint32_t)(cy + dy) * kP2);
#pragma unroll 1
            for (int dx = -1; dx <= 1; ++dx) {
                const uint32_t hsh = (((uint32_t)(cx + dx) * kP1) ^ hyz) & P.mask;
                const int i = staged ? hs_probe(S.key, hsh) : -1;
                if (i >= 0) {
                    const int c = S.count[i];
                    if (c == 0) continue;
                    bucket_hits(xi, yi, zi, self, S.start[i], c, S.off[i], loc, hit,
                                [&](int idx, int g) { body(true, idx, g); });
                } else {
                    const int2 se = __ldg(table + hsh);
                    if (se.x == -1) continue;
                    bucket_hits(xi, yi, zi, self, se.x, se.y - se.x, se.x, glob, hit,
                                [&](int idx, int g) { body(false, idx, g); });
                }
            }
        }
    }
}

// ---- CS_ComputeLambdas.glsl:108-162 ------------------------------------------------------
__global__ void __launch_bounds__(kSThreads) k_lambda_s(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, float* __restrict__ rho_out,
                                                        const int2* __restrict__ table, const uint32_t* __restrict__ lod,
                                                        uint32_t iter, const uint32_t* __restrict__ order, int cap)
{
    extern __shared__ float4 dyn[];
    __shared__ StagedShared S;
    float4* cand = dyn;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (int)__ldg(order + t) : -1;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    bool act = in;
    if (in) {
        xi = __ldg(xin + s);
        if (P.apbf && __ldg(lod + s) < iter) {
            xout[s] = xi;
            act = false;
        }
    }
    const int cx = cell_coord(xi.x, P.h), cy = cell_coord(xi.y, P.h), cz = cell_coord(xi.z, P.h);
    const bool staged =
        stage_block(P, table, S, act, cx, cy, cz, cap, [&](int k, int dst) { cand[dst] = __ldg(xin + k); });
    if (!act) return;
    auto loc = [&](int i) { return cand[i]; };
    auto glob = [&](int k) { return __ldg(xin + k); };
    float rho = P.w0_self, sg = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
    staged_walk(P, table, S, staged, xi.x, xi.y, xi.z, cx, cy, cz, s, loc, glob, [&](float r2) { return r2 <= P.h2; },
                [&](bool local, int i, int) {
                    const float4 xj = local ? cand[i] : __ldg(xin + i);
                    const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                    const float r2 = rx * rx + ry * ry + rz * rz;
                    rho += poly6_in(P, r2);
                    if (r2 >= 1e-10f) {
                        const float sc = spiky_scale(P, r2);
                        const float ax = rx * sc, ay = ry * sc, az = rz * sc;
                        sg += (ax * ax + ay * ay + az * az) * P.inv_rho0_sq;
                        gx += ax;
                        gy += ay;
                        gz += az;
                    }
                });
    gx *= P.inv_rho0;
    gy *= P.inv_rho0;
    gz *= P.inv_rho0;
    const float C = fmaxf(rho / P.rho0 - 1.0f, -P.cohesion);
    sg += gx * gx + gy * gy + gz * gz;
    xout[s] = make_float4(xi.x, xi.y, xi.z, -C / (sg + P.eps));
    rho_out[s] = rho;
}

// ---- CS_ComputeDeltaP.glsl:120-166 + CS_ApplyDeltaP.glsl:80-124 ------------------------------
__global__ void __launch_bounds__(kSThreads) k_deltap_s(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, const int2* __restrict__ table,
                                                        const uint32_t* __restrict__ lod, uint32_t iter,
                                                        const uint32_t* __restrict__ order, int cap)
{
    extern __shared__ float4 dyn[];
    __shared__ StagedShared S;
    float4* cand = dyn;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (int)__ldg(order + t) : -1;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    bool act = in;
    if (in) {
        xi = __ldg(xin + s);
        if (P.apbf && __ldg(lod + s) < iter) {
            xout[s] = xi;
            act = false;
        }
    }
    const int cx = cell_coord(xi.x, P.h), cy = cell_coord(xi.y, P.h), cz = cell_coord(xi.z, P.h);
    const bool staged =
        stage_block(P, table, S, act, cx, cy, cz, cap, [&](int k, int dst) { cand[dst] = __ldg(xin + k); });
    if (!act) return;
    auto loc = [&](int i) { return cand[i]; };
    auto glob = [&](int k) { return __ldg(xin + k); };
    const float li = xi.w;
    float dx = 0.f, dy = 0.f, dz = 0.f;
    staged_walk(P, table, S, staged, xi.x, xi.y, xi.z, cx, cy, cz, s, loc, glob,
                [&](float r2) { return r2 <= P.h2 && r2 >= 1e-10f; },
                [&](bool local, int i, int) {
                    const float4 xj = local ? cand[i] : __ldg(xin + i);
                    const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                    const float r2 = rx * rx + ry * ry + rz * rz;
                    const float sc = spiky_scale(P, r2);
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
                });
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
__global__ void __launch_bounds__(kSThreads) k_integrate_s(DevParams P, const float4* __restrict__ xs,
                                                           const float4* __restrict__ sv, float4* __restrict__ sx0,
                                                           float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ pos,
                                                           float4* __restrict__ vel, const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order, int cap)
{
    extern __shared__ float4 dyn[];
    __shared__ StagedShared S;
    float4* cand = dyn;
    float4* candv = dyn + cap;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (int)__ldg(order + t) : -1;
    float4 x4 = make_float4(0.f, 0.f, 0.f, 0.f), v0 = x4;
    if (in) {
        x4 = __ldg(xs + s);
        v0 = __ldg(sv + s);
    }
    const bool walk = in && (P.visc_on || P.vort_on);
    const int cx = cell_coord(x4.x, P.h), cy = cell_coord(x4.y, P.h), cz = cell_coord(x4.z, P.h);
    const bool staged = stage_block(P, table, S, walk, cx, cy, cz, cap, [&](int k, int dst) {
        cand[dst] = __ldg(xs + k);
        candv[dst] = __ldg(sv + k);
    });
    if (!in) return;
    float fx = 0.f, fy = 0.f, fz = 0.f, ox = 0.f, oy = 0.f, oz = 0.f;
    if (walk) {
        auto loc = [&](int i) { return cand[i]; };
        auto glob = [&](int k) { return __ldg(xs + k); };
        staged_walk(P, table, S, staged, x4.x, x4.y, x4.z, cx, cy, cz, s, loc, glob,
                    [&](float r2) { return r2 <= P.h2; },
                    [&](bool local, int i, int g) {
                        const float4 xj = local ? cand[i] : __ldg(xs + i);
                        const float rx = x4.x - xj.x, ry = x4.y - xj.y, rz = x4.z - xj.z;
                        const float r2 = rx * rx + ry * ry + rz * rz;
                        const float4 vj = local ? candv[i] : __ldg(sv + g);
                        const float ux = vj.x - v0.x, uy = vj.y - v0.y, uz = vj.z - v0.z;
                        if (P.visc_on) {
                            const float w = poly6_in(P, r2) * P.inv_rho0;
                            fx += ux * w;
                            fy += uy * w;
                            fz += uz * w;
                        }
                        if (P.vort_on && r2 >= 1e-10f) {
                            const float sc = spiky_scale(P, r2);
                            const float ax = rx * sc, ay = ry * sc, az = rz * sc;
                            ox += uy * az - uz * ay;
                            oy += uz * ax - ux * az;
                            oz += ux * ay - uy * ax;
                        }
                    });
    }
    const float4 p0 = sx0[s];
    float3 x = make_float3(x4.x, x4.y, x4.z);
    float vdx = 0.f, vdy = 0.f, vdz = 0.f;
    if (P.visc_on) {
        vdx = fx * P.viscosity;
        vdy = fy * P.viscosity;
        vdz = fz * P.viscosity;
    }
    if (P.vort_on) {
        const float wx = ox * P.inv_rho0, wy = oy * P.inv_rho0, wz = oz * P.inv_rho0;
        somega[s] = make_float4(wx, wy, wz, sqrtf(wx * wx + wy * wy + wz * wz));
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
__global__ void __launch_bounds__(kSThreads) k_vorticity_s(DevParams P, const float4* __restrict__ spos,
                                                           const float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ vel,
                                                           const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order, int cap)
{
    extern __shared__ float4 dyn[];
    __shared__ StagedShared S;
    float4* cand = dyn;  // (x, y, z, |omega|)
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = t < (int)P.n;
    const int s = in ? (int)__ldg(order + t) : -1;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (in) xi = __ldg(spos + s);
    const int cx = cell_coord(xi.x, P.h), cy = cell_coord(xi.y, P.h), cz = cell_coord(xi.z, P.h);
    const bool staged = stage_block(P, table, S, in, cx, cy, cz, cap, [&](int k, int dst) {
        const float4 p = __ldg(spos + k);
        cand[dst] = make_float4(p.x, p.y, p.z, __ldg(&somega[k].w));
    });
    if (!in) return;
    auto loc = [&](int i) { return cand[i]; };
    auto glob = [&](int k) {
        const float4 p = __ldg(spos + k);
        return make_float4(p.x, p.y, p.z, __ldg(&somega[k].w));
    };
    float ex = 0.f, ey = 0.f, ez = 0.f;
    staged_walk(P, table, S, staged, xi.x, xi.y, xi.z, cx, cy, cz, s, loc, glob,
                [&](float r2) { return r2 <= P.h2 && r2 >= 1e-10f; },
                [&](bool local, int i, int) {
                    const float4 xj = local ? cand[i] : glob(i);
                    const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                    const float r2 = rx * rx + ry * ry + rz * rz;
                    const float sc = spiky_scale(P, r2) * xj.w;
                    ex += rx * sc;
                    ey += ry * sc;
                    ez += rz * sc;
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

// staged candidates per block: 48 KB of float4 (integrate: 2 x 32 KB)
constexpr int kCapOne = 3072;
constexpr int kCapTwo = 2048;

static bool g_attr_done[64];

static void ensure_attrs(int device)
{
    if (device < 0 || device >= 64 || g_attr_done[device]) return;
    cudaFuncSetAttribute(k_lambda_s, cudaFuncAttributeMaxDynamicSharedMemorySize, kCapOne * 16);
    cudaFuncSetAttribute(k_deltap_s, cudaFuncAttributeMaxDynamicSharedMemorySize, kCapOne * 16);
    cudaFuncSetAttribute(k_vorticity_s, cudaFuncAttributeMaxDynamicSharedMemorySize, kCapOne * 16);
    cudaFuncSetAttribute(k_integrate_s, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * kCapTwo * 16);
    g_attr_done[device] = true;
}

void staged_init(int device) { ensure_attrs(device); }

static inline unsigned sgrid(uint32_t n) { return (n + kSThreads - 1) / kSThreads; }

void launch_lambda_s(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                     const uint32_t* lod, uint32_t iter, const uint32_t* order, int device, cudaStream_t st)
{
    ensure_attrs(device);
    k_lambda_s<<<sgrid(P.n), kSThreads, kCapOne * 16, st>>>(P, xin, xout, rho, table, lod, iter, order, kCapOne);
}

void launch_deltap_s(const DevParams& P, const float4* xin, float4* xout, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, int device, cudaStream_t st)
{
    ensure_attrs(device);
    k_deltap_s<<<sgrid(P.n), kSThreads, kCapOne * 16, st>>>(P, xin, xout, table, lod, iter, order, kCapOne);
}

void launch_integrate_s(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                        const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                        int device, cudaStream_t st)
{
    ensure_attrs(device);
    k_integrate_s<<<sgrid(P.n), kSThreads, 2 * kCapTwo * 16, st>>>(P, xs, sv, sx0, somega, ids, pos, vel, table, order,
                                                                     kCapTwo);
}

void launch_vorticity_s(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                        float4* vel, const int2* table, const uint32_t* order, int device, cudaStream_t st)
{
    ensure_attrs(device);
    k_vorticity_s<<<sgrid(P.n), kSThreads, kCapOne * 16, st>>>(P, spos, somega, ids, vel, table, order, kCapOne);
}

}  // namespace pbf
