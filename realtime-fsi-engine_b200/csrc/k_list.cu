// k_list.cu — neighbour mode 6: per-substep neighbour lists with a skin,
// data relabelled into Morton order.
//
// After the hash sort and the Morton sort of a substep, every per-particle
// array is gathered into processing order (label t = Morton rank), so a
// warp's own data is one coalesced run and its neighbours' data sits close by.
// The first lambda pass walks the 27 hashed buckets exactly as the reference
// does (through the hash-ordered x* of the predict) and, besides computing
// lambda, appends every candidate with r <= h + skin to the particle's list,
// in visiting order and with multiplicity: the candidate's label together
// with the index (0..26) of the bucket it came from.  Every later neighbour
// pass of the substep replays the 27 buckets from the list, applying the
// pass's own r <= h test.  This yields exactly the hits, in the order of the
// bucket walk, when
//   (a) the particle is still in the cell it was listed from (same buckets),
//   (b) it has moved at most skin/2 since the build, and
//   (c) so has every particle of the bucket: a pair left out had
//       r > h + skin at build time, so now r > h.
// Passes that move particles mark the bucket of every particle that has
// moved more than skin/2 (bucket = its predict-time hash, which is fixed for
// the substep).  A marked bucket is walked in full for everyone; a particle
// failing (a) or (b) walks all its buckets.  The visited multiset, the
// visiting order and the per-pair arithmetic (masked_body.cuh) are those of
// the bucket walk.
#include "masked_body.cuh"
#include "pbf_kernels.h"

namespace pbf {

constexpr int kLThreads = 128;
constexpr uint32_t kBucketShift = 27;  // list entry = bucket index << 27 | label
constexpr uint32_t kLabelMask = (1u << kBucketShift) - 1u;

__device__ __forceinline__ bool same_cell(const DevParams& P, float4 a, float4 b)
{
    return cell_coord(a.x, P.h) == cell_coord(b.x, P.h) && cell_coord(a.y, P.h) == cell_coord(b.y, P.h) &&
           cell_coord(a.z, P.h) == cell_coord(b.z, P.h);
}

// Calls f(b, hash) for the 27 buckets of the cell of p in walk order.
template <class F>
__device__ __forceinline__ void for_each_bucket(const DevParams& P, float4 p, F&& f)
{
    const int cx = cell_coord(p.x, P.h), cy = cell_coord(p.y, P.h), cz = cell_coord(p.z, P.h);
    int b = 0;
#pragma unroll 1
    for (int dz = -1; dz <= 1; ++dz) {
        const uint32_t hz = (uint32_t)(cz + dz) * kP3;
#pragma unroll 1
        for (int dy = -1; dy <= 1; ++dy) {
            const uint32_t hyz = hz ^ ((uint32_t)(cy + dy) * kP2);
#pragma unroll 1
            for (int dx = -1; dx <= 1; ++dx, ++b) f(b, (((uint32_t)(cx + dx) * kP1) ^ hyz) & P.mask);
        }
    }
}

// Walk of one bucket in label space (hash slot k -> label inv[k]).
template <class Hit, class Body>
__device__ __forceinline__ void walk_bucket(const ListArgs& L, uint32_t hsh, const float4* X, float4 xi, int self,
                                            Hit&& hit, Body&& body)
{
    const int2 se = __ldg(L.table + hsh);
    if (se.x == -1) return;
#pragma unroll 1
    for (int k = se.x; k < se.y; ++k) {
        const int j = (int)__ldg(L.inv + k);
        if (j == self) continue;
        const float4 xj = __ldg(X + j);
        const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
        if (hit(rx * rx + ry * ry + rz * rz)) body(j);
    }
}

// The 27 buckets walked in full (a particle that moved or changed cell).
struct FullWalk {
    const DevParams& P;
    const ListArgs& L;
    const float4* X;
    float4 xi;
    int self;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        for_each_bucket(P, xi, [&](int, uint32_t hsh) { walk_bucket(L, hsh, X, xi, self, hit, body); });
    }
};

// The list, bucket by bucket; marked buckets walked in full instead.
struct ListWalk {
    const DevParams& P;
    const ListArgs& L;
    int t;
    uint32_t cnt;
    const float4* X;
    float4 xi;
    template <class Hit, class Body>
    __device__ __forceinline__ void operator()(Hit&& hit, Body&& body) const
    {
        uint32_t c = 0;
        uint32_t e = cnt ? __ldg(L.list + t) : 0xFFFFFFFFu;  // next entry
        for_each_bucket(P, xi, [&](int b, uint32_t hsh) {
            if (__ldg(L.fastb + hsh)) {
                walk_bucket(L, hsh, X, xi, t, hit, body);
                atomicAdd(L.stats + 1, 1u);
                while (c < cnt && (e >> kBucketShift) == (uint32_t)b) {
                    ++c;
                    e = c < cnt ? __ldg(L.list + (size_t)c * P.n + t) : 0xFFFFFFFFu;
                }
                return;
            }
            while (c < cnt && (e >> kBucketShift) == (uint32_t)b) {
                const int j = (int)(e & kLabelMask);
                ++c;
                e = c < cnt ? __ldg(L.list + (size_t)c * P.n + t) : 0xFFFFFFFFu;
                const float4 xj = __ldg(X + j);
                const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                if (hit(rx * rx + ry * ry + rz * rz)) body(j);
            }
        });
    }
};

// Run core(walker) with the list when conditions (a) and (b) hold for this
// particle, else with the full bucket walk.
template <class Core>
__device__ __forceinline__ void with_walker(const DevParams& P, const ListArgs& L, const float4* X, float4 xi, int t,
                                            Core&& core)
{
    const uint32_t c = __ldg(L.cnt + t);
    const float4 b = __ldg(L.xb + t);
    const float ddx = xi.x - b.x, ddy = xi.y - b.y, ddz = xi.z - b.z;
    const float d2 = ddx * ddx + ddy * ddy + ddz * ddz;
    if (c != 0xFFFFFFFFu && d2 <= L.half_skin2 && same_cell(P, xi, b)) {
        core(ListWalk{P, L, t, c, X, xi});
    } else {
        atomicAdd(L.stats + 0, 1u);
        core(FullWalk{P, L, X, xi, t});
    }
}

// Mark the bucket of a particle that has moved more than skin/2.
__device__ __forceinline__ void mark_if_fast(const ListArgs& L, float4 x, int t)
{
    const float4 b = __ldg(L.xb + t);
    const float ddx = x.x - b.x, ddy = x.y - b.y, ddz = x.z - b.z;
    if (ddx * ddx + ddy * ddy + ddz * ddz > L.half_skin2) {
        const uint32_t k = __ldg(L.lkey + t);
        if (!L.fastb[k]) {
            L.fastb[k] = 1;
            atomicAdd(L.stats + 2, 1u);
        }
    }
}

// ---- hash slots -> Morton labels ------------------------------------------------------------
__global__ void __launch_bounds__(256) k_l_permute(uint32_t n, const uint32_t* __restrict__ order,
                                                   const uint32_t* __restrict__ ids,
                                                   const uint32_t* __restrict__ skeys, const float4* __restrict__ sx,
                                                   const float4* __restrict__ sv, const float4* __restrict__ sx0,
                                                   float4* __restrict__ lx, float4* __restrict__ lxb,
                                                   float4* __restrict__ lv, float4* __restrict__ lx0,
                                                   uint32_t* __restrict__ lid, uint32_t* __restrict__ lkey,
                                                   uint32_t* __restrict__ inv)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
        const uint32_t s = __ldg(order + t);
        const float4 x = __ldg(sx + s);
        lx[t] = x;
        lxb[t] = x;
        lv[t] = __ldg(sv + s);
        lx0[t] = __ldg(sx0 + s);
        lid[t] = __ldg(ids + s);
        lkey[t] = __ldg(skeys + s);
        inv[s] = t;
    }
}

// ---- lambda of the first iteration + list build ------------------------------------------
// The bucket walk of masked_walk (chunks of 8 tested into a hit mask), with
// the wider reach h + skin and the bucket index passed to the body.
template <class Hit, class Body>
__device__ __forceinline__ void masked_walk_b(const DevParams& P, const int2* __restrict__ table,
                                              const float4* __restrict__ X, float4 xi, int self, Hit&& hit,
                                              Body&& body)
{
    for_each_bucket(P, xi, [&](int b, uint32_t hsh) {
        const int2 se = __ldg(table + hsh);
        if (se.x == -1) return;
#pragma unroll 1
        for (int k0 = se.x; k0 < se.y; k0 += kChunk) {
            uint32_t m = 0;
#pragma unroll
            for (int c = 0; c < kChunk; ++c) {
                const int k = k0 + c;
                if (k < se.y) {
                    const float4 xj = __ldg(X + k);
                    const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
                    if (hit(rx * rx + ry * ry + rz * rz) && k != self) m |= 1u << c;
                }
            }
            while (m) {
                const int c = __ffs(m) - 1;
                m &= m - 1u;
                body(k0 + c, b);
            }
        }
    });
}

// Candidates are read from the hash-ordered x* of the predict (sx), the
// bucket layout; the list stores their labels.
__global__ void __launch_bounds__(kLThreads) k_l_lambda_build(DevParams P, const int2* __restrict__ table,
                                                              const float4* __restrict__ sx,
                                                              const uint32_t* __restrict__ order,
                                                              const uint32_t* __restrict__ inv,
                                                              const float4* __restrict__ lxb,
                                                              float4* __restrict__ lx_out, float* __restrict__ lrho,
                                                              uint32_t* __restrict__ list, uint32_t* __restrict__ cnt,
                                                              uint32_t cap, float reach2)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = (int)__ldg(order + t);
    const float4 xi = __ldg(lxb + t);
    uint32_t c = 0;
    // the lambda core sees the r <= h subset through its own hit test, in
    // the same order
    auto walk = [&](auto&& hit, auto&& body) {
        masked_walk_b(P, table, sx, xi, s, [&](float r2) { return r2 <= reach2; }, [&](int k, int b) {
            if (c < cap) list[(size_t)c * P.n + t] = ((uint32_t)b << kBucketShift) | __ldg(inv + k);
            ++c;
            const float4 xj = __ldg(sx + k);
            const float rx = xi.x - xj.x, ry = xi.y - xj.y, rz = xi.z - xj.z;
            if (hit(rx * rx + ry * ry + rz * rz)) body(k);
        });
    };
    float rho, den;
    float3 g;
    lx_out[t] = lambda_core(P, GSrc{sx}, xi, walk, rho, g, den);
    lrho[t] = rho;
    cnt[t] = c <= cap ? c : 0xFFFFFFFFu;
}

__global__ void __launch_bounds__(kLThreads) k_l_lambda(DevParams P, ListArgs L, const float4* __restrict__ lx_in,
                                                        float4* __restrict__ lx_out, float* __restrict__ lrho)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const float4 xi = __ldg(lx_in + t);
    float rho, den;
    float3 g;
    float4 out;
    with_walker(P, L, lx_in, xi, t, [&](auto&& walk) { out = lambda_core(P, GSrc{lx_in}, xi, walk, rho, g, den); });
    lx_out[t] = out;
    lrho[t] = rho;
}

__global__ void __launch_bounds__(kLThreads) k_l_deltap(DevParams P, ListArgs L, const float4* __restrict__ lx_in,
                                                        float4* __restrict__ lx_out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const float4 xi = __ldg(lx_in + t);
    float3 dp;
    float4 out;
    with_walker(P, L, lx_in, xi, t, [&](auto&& walk) { out = deltap_core(P, P.sdf, GSrc{lx_in}, xi, walk, dp); });
    lx_out[t] = out;
    mark_if_fast(L, out, t);
}

__global__ void __launch_bounds__(kLThreads) k_l_integrate(DevParams P, ListArgs L, const float4* __restrict__ lx,
                                                           const float4* __restrict__ lv, float4* __restrict__ lx0,
                                                           float4* __restrict__ lom,
                                                           const uint32_t* __restrict__ lid, float4* __restrict__ pos,
                                                           float4* __restrict__ vel)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const float4 x4 = __ldg(lx + t);
    const float4 v0 = __ldg(lv + t);
    const float4 p0 = lx0[t];
    float4 xo, vo, om;
    with_walker(P, L, lx, x4, t,
                [&](auto&& walk) { integrate_core(P, P.bmin, P.bmax, P.sdf, GSrc{lx}, GSrc{lv}, x4, v0, p0, walk, xo, vo, om); });
    if (P.vort_on) lom[t] = om;
    const uint32_t id = __ldg(lid + t);
    pos[id] = xo;
    vel[id] = vo;
    lx0[t] = xo;
    mark_if_fast(L, xo, t);
}

__global__ void __launch_bounds__(kLThreads) k_l_vorticity(DevParams P, ListArgs L, const float4* __restrict__ lx0,
                                                           const float4* __restrict__ lom,
                                                           const uint32_t* __restrict__ lid, float4* __restrict__ vel)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const float4 xi = __ldg(lx0 + t);
    float3 dv;
    bool any = false;
    with_walker(P, L, lx0, xi, t, [&](auto&& walk) { any = vorticity_core(P, GSrc{lx0}, GMag{lom}, xi, __ldg(lom + t), walk, dv); });
    if (!any) return;
    const uint32_t id = __ldg(lid + t);
    float4 v = vel[id];
    v.x += dv.x;
    v.y += dv.y;
    v.z += dv.z;
    vel[id] = v;
}

// label -> hash-slot order (for reading sorted buffers back in mode 6)
__global__ void k_l_unpermute4(uint32_t n, const uint32_t* __restrict__ inv, const float4* __restrict__ src,
                               float4* __restrict__ dst)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) dst[s] = __ldg(src + __ldg(inv + s));
}

__global__ void k_l_unpermute1(uint32_t n, const uint32_t* __restrict__ inv, const float* __restrict__ src,
                               float* __restrict__ dst)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += stride) dst[s] = __ldg(src + __ldg(inv + s));
}

// ---- launchers ------------------------------------------------------------------------------
static inline unsigned lgrid(uint32_t n) { return (n + kLThreads - 1) / kLThreads; }
static inline unsigned sgrid(uint32_t n, int sms)
{
    const uint32_t want = (n + 255u) / 256u, cap = (uint32_t)sms * 8u;
    return want < 1 ? 1 : (want > cap ? cap : want);
}

void launch_l_permute(uint32_t n, const uint32_t* order, const uint32_t* ids, const uint32_t* skeys,
                      const float4* sx, const float4* sv, const float4* sx0, float4* lx, float4* lxb, float4* lv,
                      float4* lx0, uint32_t* lid, uint32_t* lkey, uint32_t* inv, int sms, cudaStream_t st)
{
    k_l_permute<<<sgrid(n, sms), 256, 0, st>>>(n, order, ids, skeys, sx, sv, sx0, lx, lxb, lv, lx0, lid, lkey, inv);
}

void launch_l_lambda_build(const DevParams& P, const int2* table, const float4* sx, const uint32_t* order,
                           const uint32_t* inv, const float4* lxb, float4* lx_out, float* lrho, uint32_t* list,
                           uint32_t* cnt, uint32_t cap, float reach, cudaStream_t st)
{
    k_l_lambda_build<<<lgrid(P.n), kLThreads, 0, st>>>(P, table, sx, order, inv, lxb, lx_out, lrho, list, cnt, cap,
                                                       reach * reach);
}

void launch_l_lambda(const DevParams& P, const ListArgs& A, const float4* lx_in, float4* lx_out, float* lrho,
                     cudaStream_t st)
{
    k_l_lambda<<<lgrid(P.n), kLThreads, 0, st>>>(P, A, lx_in, lx_out, lrho);
}

void launch_l_deltap(const DevParams& P, const ListArgs& A, const float4* lx_in, float4* lx_out, cudaStream_t st)
{
    k_l_deltap<<<lgrid(P.n), kLThreads, 0, st>>>(P, A, lx_in, lx_out);
}

void launch_l_integrate(const DevParams& P, const ListArgs& A, const float4* lx, const float4* lv, float4* lx0,
                        float4* lom, const uint32_t* lid, float4* pos, float4* vel, cudaStream_t st)
{
    k_l_integrate<<<lgrid(P.n), kLThreads, 0, st>>>(P, A, lx, lv, lx0, lom, lid, pos, vel);
}

void launch_l_vorticity(const DevParams& P, const ListArgs& A, const float4* lx0, const float4* lom,
                        const uint32_t* lid, float4* vel, cudaStream_t st)
{
    k_l_vorticity<<<lgrid(P.n), kLThreads, 0, st>>>(P, A, lx0, lom, lid, vel);
}

void launch_l_unpermute4(uint32_t n, const uint32_t* inv, const float4* src, float4* dst, int sms, cudaStream_t st)
{
    k_l_unpermute4<<<sgrid(n, sms), 256, 0, st>>>(n, inv, src, dst);
}

void launch_l_unpermute1(uint32_t n, const uint32_t* inv, const float* src, float* dst, int sms, cudaStream_t st)
{
    k_l_unpermute1<<<sgrid(n, sms), 256, 0, st>>>(n, inv, src, dst);
}

}  // namespace pbf
