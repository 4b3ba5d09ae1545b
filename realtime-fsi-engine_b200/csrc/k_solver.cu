// k_solver.cu — the streaming per-substep passes of the PBF solver on
// sm_100a: predict + hash, the reorder into sorted float4 arrays, the cell
// table, the NaN check and the particle (un)packing.  One thread per
// particle (particle order) or per sorted slot.  The neighbour passes are
// k_masked.cu (hashed buckets) and k_dense.cu (dense cell window).
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
