// k_brick.cu — neighbour mode 7: each block stages its neighbourhood's
// buckets in shared memory through a dense cell table.
//
// A block takes 256 consecutive particles of the Morton processing order —
// about 32 cells of a compact brick of predict-time cells (the cells the
// buckets were built from, decoded from the particle's Morton code).  It
// widens their bounding box by two cells on every side and copies, for every
// cell of that box, the sorted-order bucket of the cell's hash into shared
// memory with coalesced loads (one warp per bucket); a dense table indexed by
// the cell's position in the box gives each bucket's staged range and its
// first sorted slot.  A particle whose current cell is within one cell of
// the brick (so that its 27 buckets lie in the box — after the Jacobi
// corrections most do) walks them (z outer, x inner, bucket contents in
// sorted order: the reference's visiting order, CS_ComputeLambdas.glsl:
// 126-150; a bucket reached from two colliding cells is staged and walked
// twice) from shared memory, testing chunks of 8 candidates into a hit mask
// as mode 4 does.  Any other particle, and every particle of a block whose
// box or staged total exceeds the shared-memory capacity, walks the buckets
// in global memory (mode 4's walk), so results never depend on the staging.
// Positions are staged; the integrate pass reads the neighbours' velocities
// for its hits from global memory through the staged slot index.
// Per-pair arithmetic: masked_body.cuh.
#include <climits>

#include "masked_body.cuh"
#include "pbf_kernels.h"

namespace pbf {

constexpr int kBThreads = 256;
constexpr int kBWarps = kBThreads / 32;
constexpr int kBMaxCells = 768;  // cells of the widened box
constexpr int kBCap = 3584;      // staged particles

struct BrickShared {
    int off[kBMaxCells + 1];  // staged range of box cell c: [off[c], off[c+1])
    int start[kBMaxCells];    // sorted slot of the first particle of that bucket
    int red[kBWarps][6];
    int scan[kBWarps];
    int box[6];               // x0, y0, z0, nx, ny, nz
    int fallback;
};

// Inverse of the reorder kernel's 8-bit spread (every third bit).
__device__ __forceinline__ int compact8(uint32_t v)
{
    v &= 0x00249249u;
    v = (v | (v >> 2)) & 0x000C30C3u;
    v = (v | (v >> 4)) & 0x0000F00Fu;
    v = (v | (v >> 8)) & 0x000000FFu;
    return (int)v;
}

// Predict-time cell coordinate from its low 8 bits, taking the integer
// closest to the current cell `cur` (particles move far less than 128 cells
// in a substep).
__device__ __forceinline__ int unwrap8(int low8, int cur)
{
    const int d = ((low8 - (cur & 255)) + 128) & 255;
    return cur + d - 128;
}

// Stage the buckets of the block's widened box; returns false (for the whole
// block) when they do not fit.  pc* = predict-time cell of this thread's
// particle.  `load(g, dst)` copies sorted slot g to staged index dst.
template <class Load>
__device__ __forceinline__ bool stage_brick(const DevParams& P, const int2* __restrict__ table, BrickShared& S,
                                            bool in, int pcx, int pcy, int pcz, Load&& load)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // 1. bounding box of the block's predict-time cells, widened by 2
    int v[6] = {in ? pcx : INT_MAX, in ? pcy : INT_MAX, in ? pcz : INT_MAX,
                in ? pcx : INT_MIN, in ? pcy : INT_MIN, in ? pcz : INT_MIN};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        v[a] = __reduce_min_sync(0xFFFFFFFFu, v[a]);
        v[a + 3] = __reduce_max_sync(0xFFFFFFFFu, v[a + 3]);
    }
    if (lane == 0)
#pragma unroll
        for (int a = 0; a < 6; ++a) S.red[warp][a] = v[a];
    __syncthreads();
    if (tid == 0) {
        int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
        for (int w = 0; w < kBWarps; ++w)
            for (int a = 0; a < 3; ++a) {
                lo[a] = min(lo[a], S.red[w][a]);
                hi[a] = max(hi[a], S.red[w][a + 3]);
            }
        // extents in 64-bit: cells of non-finite or scattered particles can
        // span the whole int range, which then falls back
        long long cells = 1;
        bool ok = hi[0] >= lo[0];
        for (int a = 0; a < 3; ++a) {
            const long long ext = (long long)hi[a] - (long long)lo[a] + 5;
            ok = ok && ext > 0 && ext <= kBMaxCells && lo[a] > INT_MIN + 2 && hi[a] < INT_MAX - 2;
            cells *= ok ? ext : 1;
            S.box[a] = ok ? lo[a] - 2 : 0;
            S.box[a + 3] = ok ? (int)ext : 1;
        }
        S.fallback = !ok || cells > kBMaxCells;
    }
    __syncthreads();
    if (S.fallback) return false;
    const int nx = S.box[3], ny = S.box[4], nz = S.box[5];
    const int cells = nx * ny * nz;
    // 2. bucket of every box cell, then an exclusive scan of the counts
    constexpr int kPer = (kBMaxCells + kBThreads - 1) / kBThreads;
    int cnt[kPer];
    int local = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const int c = tid * kPer + q;
        cnt[q] = 0;
        if (c < cells) {
            const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
            const uint32_t hsh = grid_hash(S.box[0] + i, S.box[1] + j, S.box[2] + k, P.mask);
            const int2 se = __ldg(table + hsh);
            S.start[c] = se.x;
            cnt[q] = se.x == -1 ? 0 : se.y - se.x;
        }
        local += cnt[q];
    }
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) S.scan[warp] = incl;
    __syncthreads();
    if (tid == 0) {
        int run = 0;
        for (int w = 0; w < kBWarps; ++w) {
            const int t = S.scan[w];
            S.scan[w] = run;
            run += t;
        }
        S.off[cells] = run;
        S.fallback = run > kBCap;
    }
    __syncthreads();
    if (S.fallback) return false;
    int base = S.scan[warp] + incl - local;
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
        const int c = tid * kPer + q;
        if (c < cells) S.off[c] = base;
        base += cnt[q];
    }
    __syncthreads();
    // 3. copy, one warp per bucket
    for (int c = warp; c < cells; c += kBWarps) {
        const int o = S.off[c], m = S.off[c + 1] - o, g = S.start[c];
        for (int l = lane; l < m; l += 32) load(g + l, o + l);
    }
    __syncthreads();
    return true;
}

// Whether a particle in cell (cx, cy, cz) has its 27 buckets in the box.
__device__ __forceinline__ bool in_box(const BrickShared& S, int cx, int cy, int cz)
{
    return cx > S.box[0] && cx < S.box[0] + S.box[3] - 1 && cy > S.box[1] && cy < S.box[1] + S.box[4] - 1 &&
           cz > S.box[2] && cz < S.box[2] + S.box[5] - 1;
}

// The 27-bucket walk over the staged copy (staged index k); self = the
// particle's sorted slot.
struct BrickWalk {
    const DevParams& P;
    const BrickShared& S;
    const float4* Xs;
    float4 xi;
    int cx, cy, cz, self;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        const int nx = S.box[3], ny = S.box[4];
        const int bx = cx - S.box[0], by = cy - S.box[1], bz = cz - S.box[2];
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                const int row = ((bz + dz) * ny + (by + dy)) * nx + bx;
#pragma unroll 1
                for (int dx = -1; dx <= 1; ++dx) {
                    const int c = row + dx;
                    const int o0 = S.off[c], o1 = S.off[c + 1];
                    const int selfk = self - S.start[c] + o0;  // staged index of self if in this bucket
#pragma unroll 1
                    for (int k0 = o0; k0 < o1; k0 += kChunk) {
                        uint32_t m = 0;
#pragma unroll
                        for (int q = 0; q < kChunk; ++q) {
                            const int k = k0 + q;
                            if (k < o1) {
                                const float4 xj = Xs[k];
                                const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                                if (hit(rx * rx + ry * ry + rz * rz) && k != selfk) m |= 1u << q;
                            }
                        }
                        while (m) {
                            const int q = __ffs(m) - 1;
                            m &= m - 1u;
                            body(k0 + q);
                        }
                    }
                }
            }
        }
    }
};

// Global data of staged entry k through the staged slot index.
struct SlotSrc {
    const int* slot;
    const float4* __restrict__ g;
    __device__ __forceinline__ float4 operator[](int k) const { return __ldg(g + slot[k]); }
};

// Thread prologue: particle, current cell, predict-time cell; stats[0]
// counts blocks and stats[1] particles that walked global memory.
#define BRICK_PROLOGUE(X)                                                                          \
    extern __shared__ float4 dyn[];                                                                \
    __shared__ BrickShared S;                                                                      \
    float4* Xs = dyn;                                                                              \
    const int t = blockIdx.x * kBThreads + threadIdx.x;                                            \
    const bool in = t < (int)P.n;                                                                  \
    const int s = in ? (int)__ldg(order + t) : 0;                                                  \
    const float4 xi = in ? __ldg(X + s) : make_float4(0.f, 0.f, 0.f, 0.f);                        \
    const int cx = cell_coord(xi.x, P.h), cy = cell_coord(xi.y, P.h), cz = cell_coord(xi.z, P.h);   \
    const uint32_t code = in ? __ldg(mcode + s) : 0u;                                              \
    const int pcx = unwrap8(compact8(code), cx), pcy = unwrap8(compact8(code >> 1), cy),            \
              pcz = unwrap8(compact8(code >> 2), cz);

#define BRICK_COUNT(staged)                                                                        \
    do {                                                                                           \
        if (stats) {                                                                               \
            if (!(staged)) {                                                                       \
                if (threadIdx.x == 0) atomicAdd(stats, 1u);                                        \
            } else {                                                                               \
                const unsigned b_ = __ballot_sync(0xFFFFFFFFu, in && !in_box(S, cx, cy, cz));      \
                if ((threadIdx.x & 31) == 0 && b_) atomicAdd(stats + 1, (unsigned)__popc(b_));     \
            }                                                                                      \
        }                                                                                          \
    } while (0)

__global__ void __launch_bounds__(kBThreads) k_lambda_b(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, float* __restrict__ rho_out,
                                                        const int2* __restrict__ table,
                                                        const uint32_t* __restrict__ lod, uint32_t iter,
                                                        const uint32_t* __restrict__ order,
                                                        const uint32_t* __restrict__ mcode,
                                                        uint32_t* __restrict__ stats)
{
    BRICK_PROLOGUE(xin)
    const bool staged = stage_brick(P, table, S, in, pcx, pcy, pcz, [&](int g, int d) { Xs[d] = __ldg(xin + g); });
    BRICK_COUNT(staged);
    if (!in) return;
    if (P.apbf && __ldg(lod + s) < iter) {
        xout[s] = xi;
        return;
    }
    float rho, den;
    float3 g;
    float4 out;
    if (staged && in_box(S, cx, cy, cz))
        out = lambda_core(P, SSrc{Xs}, xi, BrickWalk{P, S, Xs, xi, cx, cy, cz, s}, rho, g, den);
    else
        out = lambda_core(P, GSrc{xin}, xi, HashWalk{P, table, P.mask, xin, xi, s}, rho, g, den);
    xout[s] = out;
    rho_out[s] = rho;
}

__global__ void __launch_bounds__(kBThreads) k_deltap_b(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, const int2* __restrict__ table,
                                                        const uint32_t* __restrict__ lod, uint32_t iter,
                                                        const uint32_t* __restrict__ order,
                                                        const uint32_t* __restrict__ mcode,
                                                        uint32_t* __restrict__ stats)
{
    BRICK_PROLOGUE(xin)
    const bool staged = stage_brick(P, table, S, in, pcx, pcy, pcz, [&](int g, int d) { Xs[d] = __ldg(xin + g); });
    BRICK_COUNT(staged);
    if (!in) return;
    if (P.apbf && __ldg(lod + s) < iter) {
        xout[s] = xi;
        return;
    }
    float3 dp;
    if (staged && in_box(S, cx, cy, cz))
        xout[s] = deltap_core(P, P.sdf, SSrc{Xs}, xi, BrickWalk{P, S, Xs, xi, cx, cy, cz, s}, dp);
    else
        xout[s] = deltap_core(P, P.sdf, GSrc{xin}, xi, HashWalk{P, table, P.mask, xin, xi, s}, dp);
}

__global__ void __launch_bounds__(kBThreads) k_integrate_b(DevParams P, const float4* __restrict__ xs,
                                                           const float4* __restrict__ sv, float4* __restrict__ sx0,
                                                           float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ pos,
                                                           float4* __restrict__ vel, const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order,
                                                           const uint32_t* __restrict__ mcode,
                                                           uint32_t* __restrict__ stats)
{
    BRICK_PROLOGUE(xs)
    int* Ss = reinterpret_cast<int*>(dyn + kBCap);
    const bool staged = stage_brick(P, table, S, in, pcx, pcy, pcz, [&](int g, int d) {
        Xs[d] = __ldg(xs + g);
        Ss[d] = g;
    });
    BRICK_COUNT(staged);
    if (!in) return;
    const float4 v0 = __ldg(sv + s);
    const float4 p0 = sx0[s];
    float4 xo, vo, om;
    if (staged && in_box(S, cx, cy, cz))
        integrate_core(P, P.bmin, P.bmax, P.sdf, SSrc{Xs}, SlotSrc{Ss, sv}, xi, v0, p0,
                       BrickWalk{P, S, Xs, xi, cx, cy, cz, s}, xo, vo, om);
    else
        integrate_core(P, P.bmin, P.bmax, P.sdf, GSrc{xs}, GSrc{sv}, xi, v0, p0,
                       HashWalk{P, table, P.mask, xs, xi, s}, xo, vo, om);
    if (P.vort_on) somega[s] = om;
    const uint32_t id = __ldg(ids + s);
    pos[id] = xo;
    vel[id] = vo;
    sx0[s] = xo;
}

__global__ void __launch_bounds__(kBThreads) k_vorticity_b(DevParams P, const float4* __restrict__ spos,
                                                           const float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ vel,
                                                           const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order,
                                                           const uint32_t* __restrict__ mcode,
                                                           uint32_t* __restrict__ stats)
{
    BRICK_PROLOGUE(spos)
    // staged w carries the neighbour's |omega|
    const bool staged = stage_brick(P, table, S, in, pcx, pcy, pcz, [&](int g, int d) {
        const float4 p = __ldg(spos + g);
        Xs[d] = make_float4(p.x, p.y, p.z, __ldg(&somega[g].w));
    });
    BRICK_COUNT(staged);
    if (!in) return;
    float3 dv;
    bool any;
    if (staged && in_box(S, cx, cy, cz))
        any = vorticity_core(P, SSrc{Xs}, SMagW{Xs}, xi, __ldg(somega + s), BrickWalk{P, S, Xs, xi, cx, cy, cz, s}, dv);
    else
        any = vorticity_core(P, GSrc{spos}, GMag{somega}, xi, __ldg(somega + s),
                             HashWalk{P, table, P.mask, spos, xi, s}, dv);
    if (!any) return;
    const uint32_t id = __ldg(ids + s);
    float4 v = vel[id];
    v.x += dv.x;
    v.y += dv.y;
    v.z += dv.z;
    vel[id] = v;
}

// ---- launchers ---------------------------------------------------------------------------
static inline unsigned bgrid(uint32_t n) { return (n + kBThreads - 1) / kBThreads; }
constexpr size_t kBSmem1 = sizeof(float4) * kBCap;
constexpr size_t kBSmem2 = (sizeof(float4) + sizeof(int)) * kBCap;

void brick_init(int device)
{
    static bool done[64] = {};
    if (device < 0 || device >= 64 || done[device]) return;
    cudaFuncSetAttribute(k_lambda_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBSmem1);
    cudaFuncSetAttribute(k_deltap_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBSmem1);
    cudaFuncSetAttribute(k_vorticity_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBSmem1);
    cudaFuncSetAttribute(k_integrate_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBSmem2);
    done[device] = true;
}

void launch_lambda_b(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                     const uint32_t* lod, uint32_t iter, const uint32_t* order, const uint32_t* mcode,
                     uint32_t* stats, cudaStream_t st)
{
    k_lambda_b<<<bgrid(P.n), kBThreads, kBSmem1, st>>>(P, xin, xout, rho, table, lod, iter, order, mcode, stats);
}

void launch_deltap_b(const DevParams& P, const float4* xin, float4* xout, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, const uint32_t* mcode, uint32_t* stats, cudaStream_t st)
{
    k_deltap_b<<<bgrid(P.n), kBThreads, kBSmem1, st>>>(P, xin, xout, table, lod, iter, order, mcode, stats);
}

void launch_integrate_b(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                        const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                        const uint32_t* mcode, uint32_t* stats, cudaStream_t st)
{
    k_integrate_b<<<bgrid(P.n), kBThreads, kBSmem2, st>>>(P, xs, sv, sx0, somega, ids, pos, vel, table, order, mcode,
                                                          stats);
}

void launch_vorticity_b(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                        float4* vel, const int2* table, const uint32_t* order, const uint32_t* mcode,
                        uint32_t* stats, cudaStream_t st)
{
    k_vorticity_b<<<bgrid(P.n), kBThreads, kBSmem1, st>>>(P, spos, somega, ids, vel, table, order, mcode, stats);
}

}  // namespace pbf
