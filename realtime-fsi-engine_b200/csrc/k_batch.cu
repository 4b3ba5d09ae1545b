// k_batch.cu — passes of the multi-scene engine: many independent scenes of
// uneven particle counts advanced by ONE persistent launch per pass.
//
// Scenes are concatenated in HBM: scene k owns particle indices
// [off_k, off_k + n_k) and buckets [T_k, T_k + H_k) of one shared cell table.
// The predict pass writes key = T_k + hash_k(cell), so one global stable
// radix sort of the offset keys is a segmented sort: every scene's particles
// land in sorted slots [off_k, off_k + n_k), ordered within the scene by
// (hash, id) exactly as a single-scene sort orders them.  One cell-table pass
// over the sorted keys then fills every scene's buckets, with global slot
// indices.  The Morton processing order carries the scene index above the
// cell code, so thread ranges stay scene-contiguous and scene_of[t] names the
// scene of processing index t, of sorted slot t and of particle t alike.
//
// Each neighbour pass is a grid-stride loop over processing indices run by a
// grid sized to the resident capacity of the device (persistent) or one
// thread per particle; block size, persistence and the cell order are chosen
// by the engine's autotuner.  The per-particle arithmetic is the single-scene
// code of masked_body.cuh, called with the scene's table, mask, walls and SDF.
#include "masked_body.cuh"
#include "pbf_batch.h"

namespace pbf {

__device__ __forceinline__ uint32_t spread10(uint32_t v)
{
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// CS_PredictAndHash.glsl:88-130 with the scene's bucket offset added.
__global__ void __launch_bounds__(256) k_b_predict(DevParams P, const SceneDev* __restrict__ scenes,
                                                   const uint16_t* __restrict__ scene_of,
                                                   const float4* __restrict__ pos, const float4* __restrict__ vel,
                                                   uint32_t* __restrict__ keys)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += stride) {
        const SceneDev* S = scenes + __ldg(scene_of + i);
        float3 vp, xs;
        predict_particle(P, __ldg(pos + i), __ldg(vel + i), vp, xs);
        keys[i] = __ldg(&S->table_off) +
                  grid_hash(cell_coord(xs.x, P.h), cell_coord(xs.y, P.h), cell_coord(xs.z, P.h), __ldg(&S->mask));
    }
}

// Gather into sorted order (k_reorder of the single-scene engine) plus the
// scene-prefixed Morton code of the predict-time cell relative to the
// scene's lowest cell, `mbits` bits per axis.
__global__ void __launch_bounds__(256) k_b_reorder(DevParams P, const SceneDev* __restrict__ scenes,
                                                   const uint16_t* __restrict__ scene_of,
                                                   const uint32_t* __restrict__ ids, const float4* __restrict__ pos,
                                                   const float4* __restrict__ vel, float4* __restrict__ sx,
                                                   float4* __restrict__ sv, float4* __restrict__ sx0,
                                                   uint32_t* __restrict__ lod, uint32_t* __restrict__ mcode,
                                                   uint32_t mbits)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t amask = (1u << mbits) - 1u;
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
            const uint32_t k = __ldg(scene_of + s);
            const SceneDev* S = scenes + k;
            const uint32_t cx = (uint32_t)(cell_coord(xs.x, P.h) - __ldg(&S->cell_lo[0])) & amask;
            const uint32_t cy = (uint32_t)(cell_coord(xs.y, P.h) - __ldg(&S->cell_lo[1])) & amask;
            const uint32_t cz = (uint32_t)(cell_coord(xs.z, P.h) - __ldg(&S->cell_lo[2])) & amask;
            mcode[s] = (k << (3u * mbits)) | (spread10(cz) << 2) | (spread10(cy) << 1) | spread10(cx);
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

template <int B>
__global__ void __launch_bounds__(B) k_b_lambda(DevParams P, const SceneDev* __restrict__ scenes,
                                                const uint16_t* __restrict__ scene_of, const float4* __restrict__ xin,
                                                float4* __restrict__ xout, float* __restrict__ rho_out,
                                                const int2* __restrict__ table, const uint32_t* __restrict__ lod,
                                                uint32_t iter, const uint32_t* __restrict__ order)
{
    for (uint32_t t = blockIdx.x * B + threadIdx.x; t < P.n; t += gridDim.x * B) {
        const int s = order ? (int)__ldg(order + t) : (int)t;
        if (P.apbf && __ldg(lod + s) < iter) {
            xout[s] = __ldg(xin + s);
            continue;
        }
        const SceneDev* S = scenes + __ldg(scene_of + t);
        float rho;
        xout[s] = lambda_particle(P, table + __ldg(&S->table_off), __ldg(&S->mask), xin, s, rho);
        rho_out[s] = rho;
    }
}

template <int B>
__global__ void __launch_bounds__(B) k_b_deltap(DevParams P, const SceneDev* __restrict__ scenes,
                                                const uint16_t* __restrict__ scene_of, const float4* __restrict__ xin,
                                                float4* __restrict__ xout, const int2* __restrict__ table,
                                                const uint32_t* __restrict__ lod, uint32_t iter,
                                                const uint32_t* __restrict__ order)
{
    for (uint32_t t = blockIdx.x * B + threadIdx.x; t < P.n; t += gridDim.x * B) {
        const int s = order ? (int)__ldg(order + t) : (int)t;
        if (P.apbf && __ldg(lod + s) < iter) {
            xout[s] = __ldg(xin + s);
            continue;
        }
        const SceneDev* S = scenes + __ldg(scene_of + t);
        const SdfDev sdf = load_sdf(S);
        xout[s] = deltap_particle(P, table + __ldg(&S->table_off), __ldg(&S->mask), sdf, xin, s);
    }
}

template <int B>
__global__ void __launch_bounds__(B) k_b_integrate(DevParams P, const SceneDev* __restrict__ scenes,
                                                   const uint16_t* __restrict__ scene_of,
                                                   const float4* __restrict__ xs, const float4* __restrict__ sv,
                                                   float4* __restrict__ sx0, float4* __restrict__ somega,
                                                   const uint32_t* __restrict__ ids, float4* __restrict__ pos,
                                                   float4* __restrict__ vel, const int2* __restrict__ table,
                                                   const uint32_t* __restrict__ order)
{
    for (uint32_t t = blockIdx.x * B + threadIdx.x; t < P.n; t += gridDim.x * B) {
        const int s = order ? (int)__ldg(order + t) : (int)t;
        const SceneDev* S = scenes + __ldg(scene_of + t);
        const SdfDev sdf = load_sdf(S);
        float bmin[3], bmax[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            bmin[a] = __ldg(&S->bmin[a]);
            bmax[a] = __ldg(&S->bmax[a]);
        }
        integrate_particle(P, table + __ldg(&S->table_off), __ldg(&S->mask), bmin, bmax, sdf, xs, sv, sx0, somega,
                           ids, pos, vel, s);
    }
}

template <int B>
__global__ void __launch_bounds__(B) k_b_vorticity(DevParams P, const SceneDev* __restrict__ scenes,
                                                   const uint16_t* __restrict__ scene_of,
                                                   const float4* __restrict__ spos,
                                                   const float4* __restrict__ somega,
                                                   const uint32_t* __restrict__ ids, float4* __restrict__ vel,
                                                   const int2* __restrict__ table,
                                                   const uint32_t* __restrict__ order)
{
    for (uint32_t t = blockIdx.x * B + threadIdx.x; t < P.n; t += gridDim.x * B) {
        const int s = order ? (int)__ldg(order + t) : (int)t;
        const SceneDev* S = scenes + __ldg(scene_of + t);
        vorticity_particle(P, table + __ldg(&S->table_off), __ldg(&S->mask), spos, somega, ids, vel, s);
    }
}

// ---- launchers ---------------------------------------------------------------------------
static unsigned stream_blocks(uint32_t n, int sms)
{
    const uint32_t want = (n + 255u) / 256u;
    const uint32_t cap = (uint32_t)sms * 8u;
    return want < 1 ? 1 : (want > cap ? cap : want);
}

void launch_b_predict(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const float4* pos,
                      const float4* vel, uint32_t* keys, int sms, cudaStream_t st)
{
    k_b_predict<<<stream_blocks(P.n, sms), 256, 0, st>>>(P, scenes, scene_of, pos, vel, keys);
}

void launch_b_reorder(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* ids,
                      const float4* pos, const float4* vel, float4* sx, float4* sv, float4* sx0, uint32_t* lod,
                      uint32_t* mcode, uint32_t mbits, int sms, cudaStream_t st)
{
    k_b_reorder<<<stream_blocks(P.n, sms), 256, 0, st>>>(P, scenes, scene_of, ids, pos, vel, sx, sv, sx0, lod, mcode,
                                                         mbits);
}

// Grid of a neighbour pass: one thread per particle (blocks_per_sm == 0) or
// the persistent grid of sms * blocks_per_sm blocks, never more blocks than
// there are particle tiles.
static unsigned pass_blocks(uint32_t n, int block, int sms, int blocks_per_sm)
{
    const uint32_t tiles = (n + (uint32_t)block - 1u) / (uint32_t)block;
    if (blocks_per_sm <= 0) return tiles < 1 ? 1 : tiles;
    const uint32_t cap = (uint32_t)sms * (uint32_t)blocks_per_sm;
    return tiles < 1 ? 1 : (tiles < cap ? tiles : cap);
}

#define PBF_BATCH_DISPATCH(B_, KERNEL, ...)                                                           \
    switch (B_) {                                                                                     \
    case 64: KERNEL<64><<<pass_blocks(P.n, 64, L.sms, L.blocks_per_sm), 64, 0, st>>>(__VA_ARGS__); break;    \
    case 256: KERNEL<256><<<pass_blocks(P.n, 256, L.sms, L.blocks_per_sm), 256, 0, st>>>(__VA_ARGS__); break; \
    default: KERNEL<128><<<pass_blocks(P.n, 128, L.sms, L.blocks_per_sm), 128, 0, st>>>(__VA_ARGS__); break; \
    }

void launch_b_lambda(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                     const float4* xin, float4* xout, float* rho, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    PBF_BATCH_DISPATCH(L.block, k_b_lambda, P, scenes, scene_of, xin, xout, rho, table, lod, iter, order);
}

void launch_b_deltap(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                     const float4* xin, float4* xout, const int2* table, const uint32_t* lod, uint32_t iter,
                     const uint32_t* order, cudaStream_t st)
{
    PBF_BATCH_DISPATCH(L.block, k_b_deltap, P, scenes, scene_of, xin, xout, table, lod, iter, order);
}

void launch_b_integrate(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                        const float4* xs, const float4* sv, float4* sx0, float4* somega, const uint32_t* ids,
                        float4* pos, float4* vel, const int2* table, const uint32_t* order, cudaStream_t st)
{
    PBF_BATCH_DISPATCH(L.block, k_b_integrate, P, scenes, scene_of, xs, sv, sx0, somega, ids, pos, vel, table, order);
}

void launch_b_vorticity(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                        const float4* spos, const float4* somega, const uint32_t* ids, float4* vel, const int2* table,
                        const uint32_t* order, cudaStream_t st)
{
    PBF_BATCH_DISPATCH(L.block, k_b_vorticity, P, scenes, scene_of, spos, somega, ids, vel, table, order);
}

#undef PBF_BATCH_DISPATCH

// Resident blocks per SM of the heaviest pass (integrate) at block size B:
// the persistent grid the autotuner tries.
int batch_max_blocks_per_sm(int block)
{
    int nb = 0;
    switch (block) {
    case 64: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_b_integrate<64>, 64, 0); break;
    case 256: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_b_integrate<256>, 256, 0); break;
    default: cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_b_integrate<128>, 128, 0); break;
    }
    return nb < 1 ? 1 : nb;
}

}  // namespace pbf
