// k_dense.cu — neighbour mode 8: the hashed buckets replaced, where that is
// exact, by runs of a dense cell window.
//
// The scene's box plus a margin of cells on each side is a dense window.
// After the hash sort of a substep, every particle is relabelled by the
// window slot of its predict-time cell (z, then y, then x; cells outside the
// window go to one overflow slot after it for one scene, wrap into the
// scene's window in a batch) and the per-particle arrays are gathered into
// that label order.  The three x-adjacent cells of a row are then one contiguous
// label range, so a particle walks 9 runs of about 24 candidates instead of
// 27 buckets of about 8 (the reference, CS_ComputeLambdas.glsl:126-150).
//
// The run walk visits exactly the pairs of the bucket walk, in the same order,
// when for the particle's cell c
//   (a) c and its 26 neighbours lie inside the window (no wrap), and
//   (b) no cell M within Chebyshev distance 2 of c shares a hash bucket with a
//       neighbour cell N of c other than itself (M = N), and
//   (c) no particle within reach of c has moved more than 0.9 h from its
//       predict-time position while a cell sharing its predict-time cell's
//       bucket lies near enough to matter (below).
// Bucket hash(N) holds the particles of N and of every cell colliding with
// it; the reference tests them all against r <= h.  A particle that moved at
// most 0.9 h and whose predict-time cell is at Chebyshev distance >= 3 from c
// is more than 2h - 0.9h from c's box, so out of range; by (b) no other
// colliding cell is nearer.  So the in-range candidates of bucket hash(N) are
// N's own, in id order (the stable sort), and the run walk sees N's particles
// in the same order; particles of other cells wrapped into N's slot (a
// batch) are far and fail r <= h.  Within a run the cells come x - 1, x, x + 1, the
// reference's innermost loop.
//
// (b) and (c) hold or fail row by row: the argument above is about the three
// buckets of one row (dz, dy) at a time.  (a) and (b) depend only on the
// window and the hash mask: one 9-bit mask of failing rows per slot, computed
// when either changes, as is, per cell, the distance to the nearest other
// cell of its bucket.  For (c), every pass that moves particles checks each
// particle now more than 0.9 h from its predict-time position: unless that
// distance shows no colliding cell can be in a query's neighbourhood
// (settle_drift), it marks, in the window cells within 1.01 h of where the
// particle is whose neighbourhood holds a colliding cell, the row of that
// cell ("dirty" for the rest of the substep): only a query in such a cell can
// see it, and only through that row's buckets.  A particle walks the runs of
// its clean rows and the hashed buckets (through the hash-slot -> label map)
// of the others, in the reference's row order; outside the window interior
// all 27 buckets.  The walks test candidates in chunks into a hit mask and
// run the shared pair bodies of masked_body.cuh for the hits in candidate
// order, so a pair's arithmetic is the same in every walk and every mode.
// The near-zero corner of a box meets exact 32-bit collisions of the hash
// (cells (1, -1, z) and (-1, 1, z) share every bucket), so the cells along
// its three edges there always have some rows on the buckets.
//
// Work saved on top of the runs:
//   * passes after the first iteration take their threads in current-cell
//     order (a counting sort of the slots the previous pass recorded), so a
//     warp's lanes walk the same few runs;
//   * the delta-p pass replays the hit masks its iteration's lambda pass
//     recorded (same positions, same runs, same hits), and the vorticity pass
//     those of the integrate pass, except near particles the walls or the
//     SDF moved there;
//   * x/y arithmetic in packed f32x2 instructions, each lane rounded as the
//     scalar operation.
// One kernel serves one scene (B = false, constants read from the kernel
// parameters) or a batch (B = true): each scene has its own window at its own
// offset in one global slot space, and a thread takes its label's scene's hash
// mask, bucket offset, walls, SDF and window.
#include "masked_body.cuh"
#include "pbf_batch.h"
#include "pbf_kernels.h"
#include <type_traits>

namespace pbf {

constexpr int kDThreads = 128;
// The nine rows (dz, dy) of a cell's neighbourhood, bit (dz + 1) * 3 + (dy + 1).
constexpr uint32_t kAllRows = 0x1FFu;

// Batches (B = true): the scene k of a label, hash-sorted index or slot
// replaces the hash mask, walls, SDF and window of P and D with its own, so
// the code below serves one scene and many alike.
template <bool B>
__device__ __forceinline__ void scene_view(DevParams& P, DenseArgs& D, uint32_t k)
{
    if constexpr (B) {
        const SceneDev* S = D.scenes + k;
        P.mask = __ldg(&S->mask);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            P.bmin[a] = __ldg(&S->bmin[a]);
            P.bmax[a] = __ldg(&S->bmax[a]);
        }
        P.sdf = load_sdf(S);
        D.gx0 = __ldg(&S->win_g0[0]);
        D.gy0 = __ldg(&S->win_g0[1]);
        D.gz0 = __ldg(&S->win_g0[2]);
        D.nx = __ldg(&S->win_n[0]);
        D.ny = __ldg(&S->win_n[1]);
        D.nz = __ldg(&S->win_n[2]);
        D.slot0 = __ldg(&S->slot0);
        D.htable += __ldg(&S->table_off);
    }
}

template <bool B>
__device__ __forceinline__ void scene_of_label(DevParams& P, DenseArgs& D, int t)
{
    if constexpr (B) scene_view<B>(P, D, __ldg(D.scene_of + t));
}

// f(P, D) with the constants of label t's scene: the kernel's own for one
// scene (B = false, read in place), a patched copy for a batch.
template <bool B, class F>
__device__ __forceinline__ void with_scene(const DevParams& P0, const DenseArgs& D0, int t, F&& f)
{
    if constexpr (B) {
        DevParams P = P0;
        DenseArgs D = D0;
        scene_of_label<B>(P, D, t);
        f(P, D);
    } else {
        f(P0, D0);
    }
}

__device__ __forceinline__ uint32_t wrap_axis(int c, int g0, uint32_t n)
{
    const long long d = (long long)c - (long long)g0;
    if (d >= 0 && d < (long long)n) return (uint32_t)d;
    long long r = d % (long long)n;
    if (r < 0) r += (long long)n;
    return (uint32_t)r;
}

__device__ __forceinline__ uint32_t dense_key(const DenseArgs& D, int cx, int cy, int cz)
{
    return D.slot0 +
           (wrap_axis(cz, D.gz0, D.nz) * D.ny + wrap_axis(cy, D.gy0, D.ny)) * D.nx + wrap_axis(cx, D.gx0, D.nx);
}

// One scene's relabelling key of a cell: its window slot, or D.total (the
// overflow slot, after every window slot) for a cell outside the window.
// Runs never reach the overflow slot's labels; the bucket walk reaches them
// through the hash-slot -> label map like any other.
__device__ __forceinline__ uint32_t scene_key(const DenseArgs& D, int cx, int cy, int cz)
{
    const uint32_t ux = (uint32_t)cx - (uint32_t)D.gx0, uy = (uint32_t)cy - (uint32_t)D.gy0,
                   uz = (uint32_t)cz - (uint32_t)D.gz0;
    return (ux < D.nx && uy < D.ny && uz < D.nz) ? (uz * D.ny + uy) * D.nx + ux : D.total;
}

// Window slot of each hash-sorted particle's predict-time cell, x* re-derived
// from (pos, vel) of particle ids[s] exactly as the predict pass derives it.
template <bool B>
__global__ void __launch_bounds__(256) k_d_keys_pred(DevParams P0, DenseArgs D0, const uint32_t* __restrict__ ids,
                                                     const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                     uint32_t* __restrict__ dkey)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P0.n; s += stride) {
        const uint32_t id = __ldg(ids + s);
        float3 vp, xs;
        predict_particle(P0, __ldg(pos + id), __ldg(vel + id), vp, xs);
        with_scene<B>(P0, D0, (int)s, [&](const DevParams& P, const DenseArgs& D) {
            const int cx = cell_coord(xs.x, P.h), cy = cell_coord(xs.y, P.h), cz = cell_coord(xs.z, P.h);
            dkey[s] = B ? dense_key(D, cx, cy, cz) : scene_key(D, cx, cy, cz);
        });
    }
}

// The predict pass of one scene in mode 8: k_predict_hash's hash key of each
// particle's predict-time cell (particle order) and, from the same x*, the
// window slot of that cell, so that the relabelling gathers a 4-byte key by id
// instead of re-deriving x* from the particle state.
__global__ void __launch_bounds__(256) k_d_predict_hash(DevParams P, DenseArgs D, const float4* __restrict__ pos,
                                                        const float4* __restrict__ vel, uint32_t* __restrict__ keys,
                                                        uint32_t* __restrict__ dkey_id)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        float3 vp, xs;
        predict_particle(P, __ldg(pos + i), __ldg(vel + i), vp, xs);
        const int cx = cell_coord(xs.x, P.h), cy = cell_coord(xs.y, P.h), cz = cell_coord(xs.z, P.h);
        keys[i] = grid_hash(cx, cy, cz, P.mask);
        dkey_id[i] = scene_key(D, cx, cy, cz);
    }
}

// dkey[s] = the window slot of hash-sorted particle ids[s], from k_d_predict_hash.
__global__ void __launch_bounds__(256) k_d_keys_gather(uint32_t n, const uint32_t* __restrict__ ids,
                                                       const uint32_t* __restrict__ dkey_id,
                                                       uint32_t* __restrict__ dkey)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride)
        dkey[s] = __ldg(dkey_id + __ldg(ids + s));
}

// Label t = hash-sorted index order[t]: its x* (also the predict-time copy),
// predicted velocity, substep-start position, id and key, gathered from the
// particle state (the predict pass's arithmetic again), and inv[order[t]] = t.
__global__ void __launch_bounds__(256) k_d_permute(DevParams P, const uint32_t* __restrict__ order,
                                                   const uint32_t* __restrict__ ids,
                                                   const uint32_t* __restrict__ skeys,
                                                   const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                   float4* __restrict__ lx, float4* __restrict__ lxb,
                                                   float4* __restrict__ lv, float4* __restrict__ lx0,
                                                   uint32_t* __restrict__ lid, uint32_t* __restrict__ lkey,
                                                   uint32_t* __restrict__ inv)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < P.n; t += stride) {
        const uint32_t s = __ldg(order + t);
        const uint32_t id = __ldg(ids + s);
        const float4 p = __ldg(pos + id);
        const float4 v = __ldg(vel + id);
        float3 vp, xs;
        predict_particle(P, p, v, vp, xs);
        const float4 x = make_float4(xs.x, xs.y, xs.z, 0.0f);
        lx[t] = x;
        lxb[t] = x;
        lv[t] = make_float4(vp.x, vp.y, vp.z, v.w);
        lx0[t] = p;
        lid[t] = id;
        lkey[t] = __ldg(skeys + s);
        inv[s] = t;
    }
}

// The window of global slot g (its scene's, in a batch) and g's slot in it.
template <bool B>
__device__ __forceinline__ uint32_t window_of_slot(DenseArgs& D, uint32_t& mask, uint32_t g)
{
    if constexpr (B) {
        const SceneDev* S = D.scenes + __ldg(D.slot_scene + g);
        mask = __ldg(&S->mask);
        D.gx0 = __ldg(&S->win_g0[0]);
        D.gy0 = __ldg(&S->win_g0[1]);
        D.gz0 = __ldg(&S->win_g0[2]);
        D.nx = __ldg(&S->win_n[0]);
        D.ny = __ldg(&S->win_n[1]);
        D.nz = __ldg(&S->win_n[2]);
        D.slot0 = __ldg(&S->slot0);
    }
    return g - D.slot0;
}

// Conditions (a) and (b) per window slot, (b) per row: bit (dz+1)*3+(dy+1)
// is set when a neighbour cell N of that row shares its bucket with a cell
// M != N within Chebyshev distance 2; 0x1FF when the cell is at the window's
// edge (a).
template <bool B>
__global__ void __launch_bounds__(128) k_d_clean(DenseArgs D0, uint32_t mask0, uint16_t* __restrict__ clean,
                                                 uint32_t* __restrict__ unclean)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < D0.total; g += stride) {
        DenseArgs D = D0;
        uint32_t mask = mask0;
        const uint32_t s = window_of_slot<B>(D, mask, g);
        const uint32_t lx = s % D.nx, ly = (s / D.nx) % D.ny, lz = s / (D.nx * D.ny);
        uint32_t bad = kAllRows;
        if (lx >= 1 && lx + 1 < D.nx && ly >= 1 && ly + 1 < D.ny && lz >= 1 && lz + 1 < D.nz) {
            const int cx = D.gx0 + (int)lx, cy = D.gy0 + (int)ly, cz = D.gz0 + (int)lz;
            uint32_t hn[27];
#pragma unroll
            for (int u = 0; u < 27; ++u)
                hn[u] = grid_hash(cx + u % 3 - 1, cy + (u / 3) % 3 - 1, cz + u / 9 - 1, mask);
            bad = 0;
#pragma unroll 1
            for (int m = 0; m < 125; ++m) {
                const int mx = m % 5 - 2, my = (m / 5) % 5 - 2, mz = m / 25 - 2;
                const uint32_t hm = grid_hash(cx + mx, cy + my, cz + mz, mask);
                const bool inner = mx >= -1 && mx <= 1 && my >= -1 && my <= 1 && mz >= -1 && mz <= 1;
                const int self_u = inner ? (mz + 1) * 9 + (my + 1) * 3 + (mx + 1) : -1;
#pragma unroll
                for (int u = 0; u < 27; ++u)
                    if (hm == hn[u] && u != self_u) bad |= 1u << (u / 3);
            }
            if (bad) atomicAdd(unclean, 1u);
        }
        clean[g] = (uint16_t)bad;
    }
}

// Label range of the x-run centred on each window slot: slots s - 1, s, s + 1
// of one row, (-1, -1) entries being empty cells; (0, 0) when all three are
// empty and at the row ends (never walked: a walked cell is interior).
template <bool B>
__global__ void __launch_bounds__(256) k_d_runs(DenseArgs D0, const int2* __restrict__ cells, int2* __restrict__ runs)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < D0.total; g += stride) {
        DenseArgs D = D0;
        uint32_t mask = 0;
        const uint32_t ux = window_of_slot<B>(D, mask, g) % D.nx;
        int2 r = make_int2(0, 0);
        if (ux >= 1 && ux + 1 < D.nx) {
            const int2 e0 = __ldg(cells + g - 1), e1 = __ldg(cells + g), e2 = __ldg(cells + g + 1);
            const int hi = max(max(e0.y, e1.y), e2.y);
            // as unsigned, an empty cell's start (-1) is the largest
            if (hi >= 0) r = make_int2((int)min(min((uint32_t)e0.x, (uint32_t)e1.x), (uint32_t)e2.x), hi);
        }
        runs[g] = r;
    }
}

// Chebyshev distance from each window cell to the nearest other cell in the
// same hash bucket, searched up to kDcolReach (kDcolReach + 1: none that near).
constexpr int kDcolReach = 6;
template <bool B>
__global__ void __launch_bounds__(128) k_d_dcol(DenseArgs D0, uint32_t mask0, uint8_t* __restrict__ dcol)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < D0.total; g += stride) {
        DenseArgs D = D0;
        uint32_t mask = mask0;
        const uint32_t s = window_of_slot<B>(D, mask, g);
        const int cx = D.gx0 + (int)(s % D.nx), cy = D.gy0 + (int)((s / D.nx) % D.ny), cz = D.gz0 + (int)(s / (D.nx * D.ny));
        const uint32_t h0 = grid_hash(cx, cy, cz, mask);
        int best = kDcolReach + 1;
#pragma unroll 1
        for (int mz = -kDcolReach; mz <= kDcolReach; ++mz) {
#pragma unroll 1
            for (int my = -kDcolReach; my <= kDcolReach; ++my) {
                const uint32_t hyz = ((uint32_t)(cy + my) * kP2) ^ ((uint32_t)(cz + mz) * kP3);
                const int dyz = max(abs(my), abs(mz));
#pragma unroll 13
                for (int mx = -kDcolReach; mx <= kDcolReach; ++mx) {
                    const bool hit = ((((uint32_t)(cx + mx) * kP1) ^ hyz) & mask) == h0 && (mx | my | mz) != 0;
                    if (hit) best = min(best, max(dyz, abs(mx)));
                }
            }
        }
        dcol[g] = (uint8_t)best;
    }
}

// Candidates lo .. hi-1 of one hashed bucket in chunks of kChunk, tested into
// a hit mask; the body runs for the hits in candidate order (masked_walk's
// scheme).  map(k) gives the label of candidate k (the hash-slot -> label map).
struct NoRecord {
    __device__ __forceinline__ void operator()(uint32_t) const {}
};

template <int C, class Map, class Hit, class Body, class Rec = NoRecord>
__device__ __forceinline__ void masked_range(const float4* __restrict__ X, float4 xi, int self, int lo, int hi,
                                             Map&& map, Hit&& hit, Body&& body, Rec&& rec = Rec{})
{
    static_assert(C >= 1 && C <= 32, "hit mask is 32 bits");
#pragma unroll 1
    for (int k0 = lo; k0 < hi; k0 += C) {
        uint32_t m = 0;
#pragma unroll
        for (int c = 0; c < C; ++c) {
            const int k = k0 + c;
            if (k < hi) {
                const int j = map(k);
                const float4 xj = __ldg(X + j);
                const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                if (hit(rx * rx + ry * ry + rz * rz) && j != self) m |= 1u << c;
            }
        }
        rec(m);
        while (m) {
            const int c = __ffs(m) - 1;
            m &= m - 1u;
            body(map(k0 + c));
        }
    }
}

// masked_range for candidates that are labels (a run): the query's own label
// is cleared from each chunk's mask once instead of being compared with every
// candidate.
template <int C, class Hit, class Body, class Rec = NoRecord>
__device__ __forceinline__ void label_range(const float4* __restrict__ X, float4 xi, int self, int lo, int hi,
                                            Hit&& hit, Body&& body, Rec&& rec = Rec{})
{
    static_assert(C >= 4 && C <= 32 && C % 4 == 0, "hit mask is 32 bits; chunks test in quarters");
    constexpr int G = 32 / C;  // chunks tested before one drain of up to 32 candidates
    const float2 xy = make_float2(xi.x, xi.y);
#pragma unroll 1
    for (int k0 = lo; k0 < hi; k0 += G * C) {
        uint32_t m = 0;
#pragma unroll 1
        for (int g = 0; g < G; ++g) {
            const int kb = k0 + g * C;
            if (kb >= hi) break;
            uint32_t mg = 0;
            // a run's last chunk is tested only as far as the warp's lanes
            // still have candidates (in quarters of the chunk: the lanes of a
            // warp mostly share their runs): candidates past a lane's run end
            // are masked below, so the mask is the same as a whole chunk's
            const int need = (int)__reduce_max_sync(__activemask(), (uint32_t)min(hi - kb, C));
            auto test = [&](auto NC) {
                constexpr int N = decltype(NC)::value;
#pragma unroll
                for (int c = 0; c < N; ++c) {
                    const float4 xj = __ldg(X + kb + c);
                    const float2 rxy = sub_f32x2(xy, make_float2(xj.x, xj.y));
                    const float rx = rxy.x, ry = rxy.y, rz = xi.z - xj.z;
                    if (hit(rx * rx + ry * ry + rz * rz)) mg |= 1u << c;
                }
            };
            if (need > (3 * C) / 4)
                test(std::integral_constant<int, C>{});
            else if (need > C / 2)
                test(std::integral_constant<int, (3 * C) / 4>{});
            else if (need > C / 4)
                test(std::integral_constant<int, C / 2>{});
            else
                test(std::integral_constant<int, C / 4>{});
            const uint32_t ds = (uint32_t)(self - kb);
            if (ds < (uint32_t)C) mg &= ~(1u << ds);
            const int left = hi - kb;
            if (left < C) mg &= (1u << left) - 1u;
            rec(mg);
            m |= mg << (g * C);
        }
        while (m) {
            const int c = __ffs(m) - 1;
            m &= m - 1u;
            body(k0 + c);
        }
    }
}

struct InvMap {
    const uint32_t* __restrict__ inv;
    __device__ __forceinline__ int operator()(int k) const { return (int)__ldg(inv + k); }
};

// Candidates per hit mask in a run (a run holds about 24).
constexpr int kRunChunk = 16;
static_assert(kRunChunk <= kLabelPad, "a run's last chunk stays inside the padded label arrays");

// The 9 x-runs of a particle whose cell satisfies (a), (b) and (c).
struct RunWalk {
    const int2* __restrict__ runs;
    const float4* __restrict__ X;
    float4 xi;
    int self;
    int s0;  // window slot of the particle's cell
    int nx, nxy;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                const int2 r = __ldg(runs + s0 + dz * nxy + dy * nx);
                label_range<kRunChunk>(X, xi, self, r.x, r.y, hit, body);
            }
        }
    }
};

// Hit masks a lambda pass records for the delta-p pass of the same
// iteration, which reads the same positions and so walks the same runs in the
// same chunks and finds the same hits: word w of label t at hm[w * n + t], two
// 16-bit chunk masks per word in walk order; the chunk count in cnt[t], or
// kNoList when the particle walked the buckets or had more than kListChunks
// chunks.  The delta-p pass then tests only the recorded hits (for its own
// r >= 1e-10 condition) instead of every candidate.
constexpr int kListWords = kDenseListWords;
constexpr int kListChunks = 2 * kListWords;
constexpr uint8_t kNoList = 0xFF;
static_assert(kRunChunk == 16, "two chunk masks per list word");

struct RunWalkRec {
    const int2* __restrict__ runs;
    const float4* __restrict__ X;
    float4 xi;
    int self;
    int s0;
    int nx, nxy;
    uint32_t* __restrict__ hm;
    uint32_t n;
    int* chunks;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        int q = 0;
        uint32_t word = 0;
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                const int2 r = __ldg(runs + s0 + dz * nxy + dy * nx);
                label_range<kRunChunk>(X, xi, self, r.x, r.y, hit, body, [&](uint32_t m) {
                    if (q < kListChunks) {
                        if (q & 1)
                            hm[(size_t)(q >> 1) * n + self] = word | (m << 16);
                        else
                            word = m;
                    }
                    ++q;
                });
            }
        }
        if (q <= kListChunks && (q & 1)) hm[(size_t)(q >> 1) * n + self] = word;
        *chunks = q;
    }
};

struct RunWalkList {
    const int2* __restrict__ runs;
    const float4* __restrict__ X;
    float4 xi;
    int self;
    int s0;
    int nx, nxy;
    const uint32_t* __restrict__ hm;
    uint32_t n;
    __device__ __forceinline__ uint32_t chunk_mask(int q) const
    {
        const uint32_t w = __ldg(hm + (size_t)(q >> 1) * n + self);
        return (q & 1) ? (w >> 16) : (w & 0xFFFFu);
    }
    // Two consecutive chunks of a run (32 consecutive candidates) are drained
    // as one 32-bit mask: a warp then runs the pair body as many times as its
    // busiest lane has hits among 32 candidates rather than 16 twice over.
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        int q = 0;
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz) {
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                const int2 r = __ldg(runs + s0 + dz * nxy + dy * nx);
#pragma unroll 1
                for (int k0 = r.x; k0 < r.y; k0 += 2 * kRunChunk) {
                    uint32_t m;
                    if ((q & 1) == 0 && k0 + kRunChunk < r.y) {
                        m = __ldg(hm + (size_t)(q >> 1) * n + self);  // both halves belong to this run
                        q += 2;
                    } else {
                        m = chunk_mask(q++);
                        if (k0 + kRunChunk < r.y) m |= chunk_mask(q++) << 16;
                    }
                    while (m) {
                        const int c = __ffs(m) - 1;
                        m &= m - 1u;
                        const int k = k0 + c;
                        const float4 xj = __ldg(X + k);
                        // (the pair body repeats this subtraction; the two merge)
                        const float2 rxy = sub_f32x2(make_float2(xi.x, xi.y), make_float2(xj.x, xj.y));
                        const float rx = rxy.x, ry = rxy.y, rz = xi.z - xj.z;
                        // a recorded hit passed r^2 <= h^2 with these positions and this
                        // arithmetic; of the replaying passes' test (r^2 <= h^2 and
                        // r^2 >= 1e-10, delta-p and vorticity alike) the lower bound remains
                        (void)hit;
                        if (rx * rx + ry * ry + rz * rz >= 1e-10f) body(k);
                    }
                }
            }
        }
    }
};


// The 27 cells row by row in the reference's order: a row whose bit is set in
// `rows` walks its three hashed buckets (through the hash-slot -> label map),
// the others their x-run of labels.  A row's run holds the pairs of its
// buckets in the same order when (b) and (c) hold for that row, so the walk
// visits exactly the pairs of the bucket walk whatever the mask; rows =
// kAllRows is the bucket walk itself (s0 is not read then).
struct MixedWalk {
    const DevParams& P;
    const int2* __restrict__ runs;
    const int2* __restrict__ htable;
    const uint32_t* __restrict__ inv;
    const float4* __restrict__ X;
    float4 xi;
    int self;
    int s0;
    int nx, nxy;
    uint32_t rows;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        const int cx = cell_coord(xi.x, P.h), cy = cell_coord(xi.y, P.h), cz = cell_coord(xi.z, P.h);
#pragma unroll 1
        for (int dz = -1; dz <= 1; ++dz) {
            const uint32_t hz = (uint32_t)(cz + dz) * kP3;
#pragma unroll 1
            for (int dy = -1; dy <= 1; ++dy) {
                if ((rows >> ((dz + 1) * 3 + (dy + 1))) & 1u) {
                    const uint32_t hyz = hz ^ ((uint32_t)(cy + dy) * kP2);
#pragma unroll 1
                    for (int dx = -1; dx <= 1; ++dx) {
                        const int2 se = __ldg(htable + ((((uint32_t)(cx + dx) * kP1) ^ hyz) & P.mask));
                        if (se.x == -1) continue;
                        masked_range<kChunk>(X, xi, self, se.x, se.y, InvMap{inv}, hit, body);
                    }
                } else {
                    const int2 r = __ldg(runs + s0 + dz * nxy + dy * nx);
                    label_range<kRunChunk>(X, xi, self, r.x, r.y, hit, body);
                }
            }
        }
    }
};

// Window slot of the particle's current cell when its neighbourhood lies in
// the window interior (else -1); dense_rows adds the rows that (b) and (c)
// send to the buckets.
__device__ __forceinline__ int interior_slot(const DevParams& P, const DenseArgs& D, float4 xi)
{
    const uint32_t ux = (uint32_t)cell_coord(xi.x, P.h) - (uint32_t)D.gx0;
    const uint32_t uy = (uint32_t)cell_coord(xi.y, P.h) - (uint32_t)D.gy0;
    const uint32_t uz = (uint32_t)cell_coord(xi.z, P.h) - (uint32_t)D.gz0;
    if (ux - 1u < D.nx - 2u && uy - 1u < D.ny - 2u && uz - 1u < D.nz - 2u)
        return (int)(D.slot0 + (uz * D.ny + uy) * D.nx + ux);
    return -1;
}

// The interior slot (or -1) and in `rows` the rows that walk their buckets:
// those (b) or (c) rules out for runs, all of them outside the interior.
__device__ __forceinline__ int dense_rows(const DevParams& P, const DenseArgs& D, float4 xi, uint32_t& rows)
{
    const int s0 = interior_slot(P, D, xi);
    rows = s0 >= 0 ? (uint32_t)__ldg(D.clean + s0) | D.dirty[s0] : kAllRows;
    return s0;
}

__device__ __forceinline__ MixedWalk mixed_walk(const DevParams& P, const DenseArgs& D, const float4* X, float4 xi,
                                                int t, int s0, uint32_t rows)
{
    return MixedWalk{P, D.runs, D.htable, D.inv, X, xi, t, s0, (int)D.nx, (int)(D.nx * D.ny), rows};
}

__device__ __forceinline__ void count_bucket_walk(const DenseArgs& D)
{
    const uint32_t am = __activemask();
    if ((threadIdx.x & 31u) == (uint32_t)(__ffs(am) - 1)) atomicAdd(D.flag + 1, (uint32_t)__popc(am));
}

// Run core(walker) with the run walk when (a), (b) and (c) hold for every
// row, else with the mixed walk (the rows they rule out through the buckets).
template <class Core>
__device__ __forceinline__ void with_dense_walker(const DevParams& P, const DenseArgs& D, const float4* X, float4 xi,
                                                  int t, Core&& core)
{
    uint32_t rows;
    const int s0 = dense_rows(P, D, xi, rows);
    if (rows == 0) {
        core(RunWalk{D.runs, X, xi, t, s0, (int)D.nx, (int)(D.nx * D.ny)});
        return;
    }
    count_bucket_walk(D);
    core(mixed_walk(P, D, X, xi, t, s0, rows));
}

// A particle at x, predict-time position xb, that has moved more than the
// 0.9 h bound.  It can differ between the two walks only for a query whose
// neighbour cells include a cell N != M (M = its predict-time cell) with
// hash(N) = hash(M), and only if the query is within reach of x.  Such
// queries lie within Chebyshev distance 2 of x's cell (1.01 h reach), their
// neighbour cells within 3, so within 3 + cheb(cell(x), M) of M.  When M's
// nearest same-bucket cell is farther (dcol), the particle is harmless;
// otherwise every such N near the reach is found and the query cells within
// reach that hold N, but not M, in their neighbourhood get the bit of N's row
// (dz, dy) set in their dirty mask (a query holding both has a collision in
// its neighbourhood, and (b) already sends both rows to the buckets).  Kept
// out of line: it takes no registers from the passes.
__device__ __noinline__ void settle_drift(const uint8_t* dcol, uint32_t* dirty, uint32_t* count, float h, uint32_t mask,
                                          float x, float y, float z, float bx, float by, float bz, int gx0, int gy0,
                                          int gz0, uint32_t nx, uint32_t ny, uint32_t nz)
{
    const float c[3] = {x, y, z}, cb[3] = {bx, by, bz};
    const int g0[3] = {gx0, gy0, gz0};
    const uint32_t nd[3] = {nx, ny, nz};
    long long m[3], rl[3], rh[3], cheb = 0;
    uint32_t um[3];
    bool inside = true;
    const float r = 1.01f * h;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        m[a] = cell_coord(cb[a], h);
        const long long d = (long long)cell_coord(c[a], h) - m[a];
        cheb = max(cheb, d < 0 ? -d : d);
        um[a] = (uint32_t)m[a] - (uint32_t)g0[a];
        inside = inside && um[a] < nd[a];
        rl[a] = cell_coord(c[a] - r, h);
        rh[a] = min((long long)cell_coord(c[a] + r, h), rl[a] + 3);
    }
    if (inside && cheb + 3 < (long long)dcol[(um[2] * ny + um[1]) * nx + um[0]]) return;
    // Queries affected: cells q within reach of x whose neighbourhood holds
    // a cell N != M of M's bucket but not M itself.  N then lies within one
    // cell of the reach box.
    const uint32_t hm = grid_hash((int)m[0], (int)m[1], (int)m[2], mask);
    bool marked = false;
    for (long long qz = rl[2] - 1; qz <= rh[2] + 1; ++qz)
        for (long long qy = rl[1] - 1; qy <= rh[1] + 1; ++qy)
            for (long long qx = rl[0] - 1; qx <= rh[0] + 1; ++qx) {
                if ((qx == m[0] && qy == m[1] && qz == m[2]) ||
                    grid_hash((int)(uint32_t)qx, (int)(uint32_t)qy, (int)(uint32_t)qz, mask) != hm)
                    continue;
                // N = (qx, qy, qz): mark reach cells within one cell of N and
                // more than one cell from M
                for (long long cz = max(rl[2], qz - 1); cz <= min(rh[2], qz + 1); ++cz)
                    for (long long cy = max(rl[1], qy - 1); cy <= min(rh[1], qy + 1); ++cy)
                        for (long long cx = max(rl[0], qx - 1); cx <= min(rh[0], qx + 1); ++cx) {
                            const long long dm = max(max(cx - m[0], m[0] - cx), max(max(cy - m[1], m[1] - cy),
                                                                                   max(cz - m[2], m[2] - cz)));
                            if (dm <= 1) continue;
                            const uint32_t ux = (uint32_t)cx - (uint32_t)g0[0], uy = (uint32_t)cy - (uint32_t)g0[1],
                                           uz = (uint32_t)cz - (uint32_t)g0[2];
                            if (ux < nx && uy < ny && uz < nz)
                                atomicOr(dirty + (uz * ny + uy) * nx + ux, 1u << (int)((qz - cz + 1) * 3 + (qy - cy + 1)));
                            marked = true;
                        }
            }
    if (marked) atomicAdd(count, 1u);
}

__device__ __forceinline__ void check_drift(const DevParams& P, const DenseArgs& D, float4 x, int t)
{
    const float4 b = __ldg(D.xb + t);
    const float dx = x.x - b.x, dy = x.y - b.y, dz = x.z - b.z;
    // NaN positions count as moved (the comparison is false for NaN)
    if (!(dx * dx + dy * dy + dz * dz <= D.drift2))
        settle_drift(D.dcol + D.slot0, D.dirty + D.slot0, D.flag, P.h, P.mask, x.x, x.y, x.z, b.x, b.y, b.z, D.gx0,
                     D.gy0, D.gz0, D.nx, D.ny, D.nz);
}

// Label t moved in the integrate pass: the queries whose runs hold it (the 27
// window cells around its label's slot) must walk, not replay, in the
// vorticity pass.
__device__ __forceinline__ void mark_moved(const DevParams& P, const DenseArgs& D, int t)
{
    const float4 b = __ldg(D.xb + t);
    const int ux = (int)wrap_axis(cell_coord(b.x, P.h), D.gx0, D.nx);
    const int uy = (int)wrap_axis(cell_coord(b.y, P.h), D.gy0, D.ny);
    const int uz = (int)wrap_axis(cell_coord(b.z, P.h), D.gz0, D.nz);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = ux + dx, y = uy + dy, z = uz + dz;
                if (x >= 0 && x < (int)D.nx && y >= 0 && y < (int)D.ny && z >= 0 && z < (int)D.nz)
                    D.vmark[D.slot0 + ((uint32_t)z * D.ny + (uint32_t)y) * D.nx + (uint32_t)x] = 1;
            }
}

// Label-order arrays gathered back into hash-sorted order (slot s <- label
// inv[s]) for the buffer reads of the stage-level API.
__global__ void k_d_unpermute4(uint32_t n, const uint32_t* __restrict__ inv, const float4* __restrict__ src,
                               float4* __restrict__ dst)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) dst[s] = __ldg(src + __ldg(inv + s));
}

__global__ void k_d_unpermute1(uint32_t n, const uint32_t* __restrict__ inv, const float* __restrict__ src,
                               float* __restrict__ dst)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) dst[s] = __ldg(src + __ldg(inv + s));
}

// ---- thread order by current cell ----------------------------------------------------------
// The labels follow the predict-time cells; once the corrections have moved
// particles, consecutive labels query different current cells and a warp's
// candidate loads scatter.  Before a pass whose particles have moved, labels
// are bucketed by the window slot of their current cell (counting sort: count,
// scan, place); the pass's thread i then takes label order[i].  The order only
// changes which thread computes which particle, never a result, so the place
// step may use atomics in any order.
constexpr uint32_t kScanItems = 4096;  // counters per block of the slot scan

// Runs of equal slots among the lanes of a warp (lanes hold consecutive
// labels, mostly of one cell): the lane that heads this lane's run and the
// run's length.
__device__ __forceinline__ void slot_run(uint32_t s, uint32_t lane, uint32_t& head, uint32_t& len)
{
    const uint32_t prev = __shfl_up_sync(0xffffffffu, s, 1);
    const uint32_t heads = __ballot_sync(0xffffffffu, lane == 0u || prev != s);
    head = 31u - (uint32_t)__clz(heads & (0xffffffffu >> (31u - lane)));
    const uint32_t after = heads & ~(0xffffffffu >> (31u - head));
    len = (after ? (uint32_t)(__ffs(after) - 1) : 32u) - head;
}

constexpr uint32_t kNoSlot = 0xffffffffu;

// Global slot of the cell of x (cells outside the window: the extra slot D.total).
__device__ __forceinline__ uint32_t current_slot(const DevParams& P, const DenseArgs& D, float4 x)
{
    const uint32_t ux = (uint32_t)cell_coord(x.x, P.h) - (uint32_t)D.gx0;
    const uint32_t uy = (uint32_t)cell_coord(x.y, P.h) - (uint32_t)D.gy0;
    const uint32_t uz = (uint32_t)cell_coord(x.z, P.h) - (uint32_t)D.gz0;
    return (ux < D.nx && uy < D.ny && uz < D.nz) ? D.slot0 + (uz * D.ny + uy) * D.nx + ux : D.total;
}

// slot of the current cell
template <bool B>
__global__ void __launch_bounds__(256) k_d_cslot(DevParams P0, DenseArgs D0, const float4* __restrict__ X,
                                                 uint32_t* __restrict__ slot_of, uint32_t* __restrict__ cnt)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t s = kNoSlot;
    if (t < P0.n) {
        with_scene<B>(P0, D0, (int)t,
                      [&](const DevParams& P, const DenseArgs& D) { s = current_slot(P, D, __ldg(X + t)); });
        slot_of[t] = s;
    }
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t head, len;
    slot_run(s, lane, head, len);
    if (lane == head && s != kNoSlot) atomicAdd(cnt + s, len);
}

// The slot a pass's output position falls in, recorded for the thread order
// of the next pass (k_d_cslot's work folded into the pass that moves the
// particle).  Every lane of the warp calls it; valid = the lane has a particle.
__device__ __forceinline__ void record_slot(const DevParams& P, const DenseArgs& D, float4 x, int t, bool valid)
{
    uint32_t s = kNoSlot;
    if (valid) {
        s = current_slot(P, D, x);
        D.rec_slot[t] = s;
    }
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t head, len;
    slot_run(s, lane, head, len);
    if (lane == head && s != kNoSlot) atomicAdd(D.rec_cnt + s, len);
}

// exclusive scan of cnt[0 .. m) in place: per block of kScanItems, then the
// block sums, then the block offsets
__global__ void __launch_bounds__(1024) k_d_scan_blocks(uint32_t* __restrict__ cnt, uint32_t m,
                                                        uint32_t* __restrict__ block_sums)
{
    __shared__ uint32_t warp_sums[32];
    const uint32_t base = blockIdx.x * kScanItems + threadIdx.x * 4u;
    uint32_t v[4], local = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = base + k < m ? cnt[base + k] : 0u;
        local += v[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t run = incl - local + (warp ? warp_sums[warp - 1] : 0u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (base + k < m) cnt[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == 1023) block_sums[blockIdx.x] = warp_sums[31];
}

__global__ void __launch_bounds__(1024) k_d_scan_sums(uint32_t* __restrict__ block_sums, uint32_t nb)
{
    __shared__ uint32_t warp_sums[32];
    const uint32_t chunk = (nb + 1023u) / 1024u;
    const uint32_t begin = threadIdx.x * chunk, end = min(begin + chunk, nb);
    uint32_t local = 0;
    for (uint32_t i = begin; i < end; ++i) local += block_sums[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
    }
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sums[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        warp_sums[lane] = w;
    }
    __syncthreads();
    uint32_t run = incl - local + (warp ? warp_sums[warp - 1] : 0u);
    for (uint32_t i = begin; i < end; ++i) {
        const uint32_t v = block_sums[i];
        block_sums[i] = run;
        run += v;
    }
}

__global__ void __launch_bounds__(256) k_d_place(uint32_t n, const uint32_t* __restrict__ slot_of,
                                                 uint32_t* __restrict__ start, const uint32_t* __restrict__ block_offs,
                                                 uint32_t* __restrict__ order)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = t < n ? __ldg(slot_of + t) : kNoSlot;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t head, len;
    slot_run(s, lane, head, len);
    uint32_t b = 0;
    if (lane == head && s != kNoSlot) b = atomicAdd(start + s, len);
    b = __shfl_sync(0xffffffffu, b, head);
    if (s != kNoSlot) order[__ldg(block_offs + s / kScanItems) + b + (lane - head)] = t;
}

// ---- relabelling of one scene by counting -----------------------------------------------
// Labels in the order of a stable sort of the hash-sorted sequence by slot
// key, without the sort: within the window a cell has one hash, so all its
// particles lie in one bucket's range of the hash sort, in id order, and a
// particle's label is the start of its slot (a counting scan over the slots)
// plus the number of particles of the same slot before it in that range.
// The overflow slot's particles (cells outside the window, from several
// buckets) are placed in any order: runs never reach them, and everything
// else they take part in follows the hash-sorted order through `inv`.
__global__ void __launch_bounds__(256) k_d_relabel_count(uint32_t n, const uint32_t* __restrict__ dkey,
                                                         uint32_t* __restrict__ cnt)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t k = s < n ? __ldg(dkey + s) : kNoSlot;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t head, len;
    slot_run(k, lane, head, len);
    if (lane == head && k != kNoSlot) atomicAdd(cnt + k, len);
}

__global__ void __launch_bounds__(256) k_d_relabel_place(uint32_t n, const uint32_t* __restrict__ dkey,
                                                         const uint32_t* __restrict__ skeys,
                                                         const uint32_t* __restrict__ start,
                                                         const uint32_t* __restrict__ block_offs, uint32_t overflow,
                                                         uint32_t* __restrict__ overflow_count,
                                                         uint32_t* __restrict__ order, uint32_t* __restrict__ sorted_keys)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) {
        const uint32_t k = __ldg(dkey + s);
        uint32_t r = 0;
        if (k == overflow) {
            r = atomicAdd(overflow_count, 1u);
        } else {
            // earlier particles of this slot in this bucket's range
            const uint32_t hk = __ldg(skeys + s);
            for (uint32_t q = s; q > 0 && __ldg(skeys + q - 1) == hk; --q) r += __ldg(dkey + q - 1) == k ? 1u : 0u;
        }
        const uint32_t t = __ldg(block_offs + k / kScanItems) + __ldg(start + k) + r;
        order[t] = s;
        sorted_keys[t] = k;
    }
}

// 10 resident blocks (48 registers, 8 bytes spilled): with the s_corr sum of
// the delta-p pass in its pair body, 12 blocks (40 registers, 132 bytes
// spilled) took 1.225 ms per 4M launch against 1.165.  The pass also writes
// each particle's lambda-independent delta-p part (DevParams::dpb).
template <bool B>
__global__ void __launch_bounds__(kDThreads, 10) k_d_lambda(DevParams P0, DenseArgs D0, const float4* __restrict__ lx_in,
                                                            float4* __restrict__ lx_out, float* __restrict__ lrho)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int)P0.n) return;
    const int t = D0.order ? (int)__ldg(D0.order + i) : i;
    with_scene<B>(P0, D0, t, [&](const DevParams& P, const DenseArgs& D) {
        const float4 xi = __ldg(lx_in + t);
        float rho, den;
        float3 g;
        float4 out;
        uint32_t rows;
        const int s0 = dense_rows(P, D, xi, rows);
        float3 b;
        if (rows == 0) {
            int q = 0;
            out = lambda_core(P, GSrc{lx_in}, xi,
                              RunWalkRec{D.runs, lx_in, xi, t, s0, (int)D.nx, (int)(D.nx * D.ny), D.hm, P.n, &q}, rho, g,
                              den, b);
            D.hcnt[t] = q <= kListChunks ? (uint8_t)q : kNoList;
        } else {
            count_bucket_walk(D);
            out = lambda_core(P, GSrc{lx_in}, xi, mixed_walk(P, D, lx_in, xi, t, s0, rows), rho, g, den, b);
            D.hcnt[t] = kNoList;
        }
        lx_out[t] = out;
        lrho[t] = rho;
        P.dpb[t] = make_float4(b.x, b.y, b.z, 0.f);
    });
}

// 16 resident blocks (32 registers, spills on the SDF projection's path): the
// replay's pair bodies, which load and scale only lambda_j, wait on their
// neighbour loads, and the extra warps hide more of that than the spills cost
// (12 blocks: 0.758 ms per 4M launch, 16: 0.731).
template <bool B>
__global__ void __launch_bounds__(kDThreads, 16) k_d_deltap(DevParams P0, DenseArgs D0, const float4* __restrict__ lx_in,
                                                            float4* __restrict__ lx_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < (int)P0.n;
    const int t = live ? (D0.order ? (int)__ldg(D0.order + i) : i) : 0;
    with_scene<B>(P0, D0, t, [&](const DevParams& P, const DenseArgs& D) {
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            const float4 xi = __ldg(lx_in + t);
            const float4 b4 = __ldg(P.dpb + t);
            const float3 b = make_float3(b4.x, b4.y, b4.z);
            float3 dp;
            if (D.use_list && __ldg(D.hcnt + t) != kNoList) {
                // the lambda pass of this iteration walked this particle's runs
                const int s0 = interior_slot(P, D, xi);
                out = deltap_core(P, P.sdf, GSrc{lx_in}, xi,
                                  RunWalkList{D.runs, lx_in, xi, t, s0, (int)D.nx, (int)(D.nx * D.ny), D.hm, P.n}, dp,
                                  b);
            } else {
                with_dense_walker(P, D, lx_in, xi, t,
                                  [&](auto&& walk) { out = deltap_core(P, P.sdf, GSrc{lx_in}, xi, walk, dp, b); });
            }
            lx_out[t] = out;
            check_drift(P, D, out, t);
        }
        if (D.rec_cnt) record_slot(P, D, out, t, live);
    });
}

template <bool B, bool R>
__global__ void __launch_bounds__(kDThreads, 10) k_d_integrate(DevParams P0, DenseArgs D0, const float4* __restrict__ lx,
                                                           const float4* __restrict__ lv, float4* __restrict__ lx0,
                                                           float4* __restrict__ lom,
                                                           const uint32_t* __restrict__ lid, float4* __restrict__ pos,
                                                           float4* __restrict__ vel)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < (int)P0.n;
    const int t = live ? (D0.order ? (int)__ldg(D0.order + i) : i) : 0;
    with_scene<B>(P0, D0, t, [&](const DevParams& P, const DenseArgs& D) {
        float4 xo = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            const float4 x4 = __ldg(lx + t);
            const float4 v0 = __ldg(lv + t);
            float4 vo, om;
            auto core = [&](auto&& walk) {
                integrate_core(P, P.bmin, P.bmax, P.sdf, GSrc{lx}, GSrc{lv}, x4, v0, [&] { return lx0[t]; }, walk, xo,
                               vo, om);
            };
            if constexpr (R) {
                // the vorticity pass walks the committed positions, equal to
                // x* unless the walls or the SDF moved the particle: record
                // the hit masks, and where a particle moved, mark the query
                // cells whose runs hold it
                uint32_t rows;
                const int s0 = dense_rows(P, D, x4, rows);
                if (rows == 0) {
                    int q = 0;
                    core(RunWalkRec{D.runs, lx, x4, t, s0, (int)D.nx, (int)(D.nx * D.ny), D.hm, P.n, &q});
                    D.hcnt[t] = q <= kListChunks ? (uint8_t)q : kNoList;
                } else {
                    count_bucket_walk(D);
                    core(mixed_walk(P, D, lx, x4, t, s0, rows));
                    D.hcnt[t] = kNoList;
                }
                if (xo.x != x4.x || xo.y != x4.y || xo.z != x4.z) {
                    D.hcnt[t] = kNoList;
                    mark_moved(P, D, t);
                }
            } else {
                with_dense_walker(P, D, lx, x4, t, core);
            }
            if (P.vort_on) lom[t] = om;
            const uint32_t id = __ldg(lid + t);
            pos[id] = xo;
            vel[id] = vo;
            // (the committed position carries |omega| in w for the vorticity
            // pass, which then reads a neighbour's position and |omega| in one load)
            lx0[t] = P.vort_on ? make_float4(xo.x, xo.y, xo.z, om.w) : xo;
            check_drift(P, D, xo, t);
        }
        if (D.rec_cnt) record_slot(P, D, xo, t, live);
    });
}

template <bool B>
__global__ void __launch_bounds__(kDThreads, 12) k_d_vorticity(DevParams P0, DenseArgs D0, const float4* __restrict__ lx0,
                                                           const float4* __restrict__ lom,
                                                           const uint32_t* __restrict__ lid, float4* __restrict__ vel)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int)P0.n) return;
    const int t = D0.order ? (int)__ldg(D0.order + i) : i;
    with_scene<B>(P0, D0, t, [&](const DevParams& P, const DenseArgs& D) {
        const float4 xi = __ldg(lx0 + t);
        float3 dv;
        bool any = false;
        auto core = [&](auto&& walk) {
            any = vorticity_core(P, GSrc{lx0}, GMagX{lx0}, xi, [&] { return __ldg(lom + t); }, walk, dv);
        };
        const int s0 = D.use_list && __ldg(D.hcnt + t) != kNoList ? interior_slot(P, D, xi) : -1;
        if (s0 >= 0 && !D.vmark[s0])
            // integrate walked this particle's runs over the same positions
            core(RunWalkList{D.runs, lx0, xi, t, s0, (int)D.nx, (int)(D.nx * D.ny), D.hm, P.n});
        else
            with_dense_walker(P, D, lx0, xi, t, core);
        if (!any) return;
        const uint32_t id = __ldg(lid + t);
        float4 v = vel[id];
        v.x += dv.x;
        v.y += dv.y;
        v.z += dv.z;
        vel[id] = v;
    });
}

// ---- launchers ------------------------------------------------------------------------------
static inline unsigned dgrid(uint32_t n) { return (n + kDThreads - 1) / kDThreads; }
static inline unsigned capped_grid(uint32_t n, uint32_t threads, int sms, uint32_t per_sm)
{
    const uint32_t want = (n + threads - 1u) / threads, cap = (uint32_t)sms * per_sm;
    return want < 1 ? 1 : (want > cap ? cap : want);
}

// B = true for the scenes of a batch
#define PBF_DENSE_LAUNCH(KERNEL, GRID, BLOCK, ...)                                                 \
    do {                                                                                          \
        if (D.scenes)                                                                             \
            KERNEL<true><<<(GRID), (BLOCK), 0, st>>>(__VA_ARGS__);                                \
        else                                                                                      \
            KERNEL<false><<<(GRID), (BLOCK), 0, st>>>(__VA_ARGS__);                               \
    } while (0)

void launch_d_keys_pred(const DevParams& P, const DenseArgs& D, const uint32_t* ids, const float4* pos,
                        const float4* vel, uint32_t* dkey, int sms, cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_keys_pred, capped_grid(P.n, 256, sms, 8), 256, P, D, ids, pos, vel, dkey);
}

void launch_d_predict_hash(const DevParams& P, const DenseArgs& D, const float4* pos, const float4* vel,
                           uint32_t* keys, uint32_t* dkey_id, int sms, cudaStream_t st)
{
    k_d_predict_hash<<<capped_grid(P.n, 256, sms, 8), 256, 0, st>>>(P, D, pos, vel, keys, dkey_id);
}

void launch_d_keys_gather(uint32_t n, const uint32_t* ids, const uint32_t* dkey_id, uint32_t* dkey, int sms,
                          cudaStream_t st)
{
    k_d_keys_gather<<<capped_grid(n, 256, sms, 8), 256, 0, st>>>(n, ids, dkey_id, dkey);
}

void launch_d_permute(const DevParams& P, const uint32_t* order, const uint32_t* ids, const uint32_t* skeys,
                      const float4* pos, const float4* vel, float4* lx, float4* lxb, float4* lv, float4* lx0,
                      uint32_t* lid, uint32_t* lkey, uint32_t* inv, int sms, cudaStream_t st)
{
    k_d_permute<<<capped_grid(P.n, 256, sms, 8), 256, 0, st>>>(P, order, ids, skeys, pos, vel, lx, lxb, lv, lx0, lid,
                                                               lkey, inv);
}

void launch_d_clean(const DenseArgs& D, uint32_t mask, uint16_t* clean, uint32_t* unclean, int sms, cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_clean, capped_grid(D.total, 128, sms, 16), 128, D, mask, clean, unclean);
}

void launch_d_runs(const DenseArgs& D, const int2* cells, int2* runs, int sms, cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_runs, capped_grid(D.total, 256, sms, 8), 256, D, cells, runs);
}

void launch_d_dcol(const DenseArgs& D, uint32_t mask, uint8_t* dcol, int sms, cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_dcol, capped_grid(D.total, 128, sms, 16), 128, D, mask, dcol);
}

uint32_t order_scan_blocks(uint32_t slots) { return (slots + 1u + kScanItems - 1u) / kScanItems; }

void launch_d_order(const DevParams& P, const DenseArgs& D, const float4* X, uint32_t* slot_of, uint32_t* cnt,
                    uint32_t* block_sums, uint32_t* order, cudaStream_t st, uint64_t* launches)
{
    const uint32_t m = D.total + 1u;  // slots + the outside slot
    const uint32_t nb = order_scan_blocks(D.total);
    cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * m, st);
    const unsigned g = (P.n + 255u) / 256u;
    PBF_DENSE_LAUNCH(k_d_cslot, g, 256, P, D, X, slot_of, cnt);
    k_d_scan_blocks<<<nb, 1024, 0, st>>>(cnt, m, block_sums);
    k_d_scan_sums<<<1, 1024, 0, st>>>(block_sums, nb);
    k_d_place<<<g, 256, 0, st>>>(P.n, slot_of, cnt, block_sums, order);
    *launches += 4;
}

void launch_d_relabel(uint32_t n, uint32_t slots, const uint32_t* dkey, const uint32_t* skeys, uint32_t* cnt,
                      uint32_t* block_sums, uint32_t* overflow_count, uint32_t* order, uint32_t* sorted_keys, int sms,
                      cudaStream_t st, uint64_t* launches)
{
    const uint32_t m = slots + 1u;  // window slots + the overflow slot
    const uint32_t nb = order_scan_blocks(slots);
    cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * m, st);
    cudaMemsetAsync(overflow_count, 0, sizeof(uint32_t), st);
    k_d_relabel_count<<<(n + 255u) / 256u, 256, 0, st>>>(n, dkey, cnt);
    k_d_scan_blocks<<<nb, 1024, 0, st>>>(cnt, m, block_sums);
    k_d_scan_sums<<<1, 1024, 0, st>>>(block_sums, nb);
    k_d_relabel_place<<<capped_grid(n, 256, sms, 8), 256, 0, st>>>(n, dkey, skeys, cnt, block_sums, slots,
                                                                  overflow_count, order, sorted_keys);
    *launches += 4;
}

void launch_d_order_recorded(const DevParams& P, const DenseArgs& D, const uint32_t* slot_of, uint32_t* cnt,
                             uint32_t* block_sums, uint32_t* order, cudaStream_t st, uint64_t* launches)
{
    const uint32_t m = D.total + 1u;
    const uint32_t nb = order_scan_blocks(D.total);
    const unsigned g = (P.n + 255u) / 256u;
    k_d_scan_blocks<<<nb, 1024, 0, st>>>(cnt, m, block_sums);
    k_d_scan_sums<<<1, 1024, 0, st>>>(block_sums, nb);
    k_d_place<<<g, 256, 0, st>>>(P.n, slot_of, cnt, block_sums, order);
    *launches += 3;
}

void launch_d_lambda(const DevParams& P, const DenseArgs& D, const float4* lx_in, float4* lx_out, float* lrho,
                     cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_lambda, dgrid(P.n), kDThreads, P, D, lx_in, lx_out, lrho);
}

void launch_d_deltap(const DevParams& P, const DenseArgs& D, const float4* lx_in, float4* lx_out, cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_deltap, dgrid(P.n), kDThreads, P, D, lx_in, lx_out);
}

void launch_d_integrate(const DevParams& P, const DenseArgs& D, const float4* lx, const float4* lv, float4* lx0,
                        float4* lom, const uint32_t* lid, float4* pos, float4* vel, cudaStream_t st)
{
    // R: record hit masks for the vorticity pass
    if (D.rec_list) {
        if (D.scenes)
            k_d_integrate<true, true><<<dgrid(P.n), kDThreads, 0, st>>>(P, D, lx, lv, lx0, lom, lid, pos, vel);
        else
            k_d_integrate<false, true><<<dgrid(P.n), kDThreads, 0, st>>>(P, D, lx, lv, lx0, lom, lid, pos, vel);
    } else {
        if (D.scenes)
            k_d_integrate<true, false><<<dgrid(P.n), kDThreads, 0, st>>>(P, D, lx, lv, lx0, lom, lid, pos, vel);
        else
            k_d_integrate<false, false><<<dgrid(P.n), kDThreads, 0, st>>>(P, D, lx, lv, lx0, lom, lid, pos, vel);
    }
}

void launch_d_vorticity(const DevParams& P, const DenseArgs& D, const float4* lx0, const float4* lom,
                        const uint32_t* lid, float4* vel, cudaStream_t st)
{
    PBF_DENSE_LAUNCH(k_d_vorticity, dgrid(P.n), kDThreads, P, D, lx0, lom, lid, vel);
}

#undef PBF_DENSE_LAUNCH

void launch_d_unpermute4(uint32_t n, const uint32_t* inv, const float4* src, float4* dst, int sms, cudaStream_t st)
{
    const uint32_t want = (n + 255u) / 256u, cap = (uint32_t)sms * 8u;
    k_d_unpermute4<<<want < 1 ? 1 : (want > cap ? cap : want), 256, 0, st>>>(n, inv, src, dst);
}

void launch_d_unpermute1(uint32_t n, const uint32_t* inv, const float* src, float* dst, int sms, cudaStream_t st)
{
    const uint32_t want = (n + 255u) / 256u, cap = (uint32_t)sms * 8u;
    k_d_unpermute1<<<want < 1 ? 1 : (want > cap ? cap : want), 256, 0, st>>>(n, inv, src, dst);
}

}  // namespace pbf
