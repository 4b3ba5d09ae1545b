// k_sdf.cu — SDF grid utilities and the contact pre-filter.
#include "pbf_kernels.h"

namespace pbf {

// Minimum of each of the six boundary faces of the grid (used for the exact
// far-obstacle skip in sdf_project).  One block per face.
__global__ void k_sdf_slab_min(const float* __restrict__ dist, int dx, int dy, int dz, float* __restrict__ out)
{
    const int face = blockIdx.x;  // 0:x=0 1:x=dx-1 2:y=0 3:y=dy-1 4:z=0 5:z=dz-1
    const int axis = face >> 1;
    const int fixed = (face & 1) ? (axis == 0 ? dx - 1 : (axis == 1 ? dy - 1 : dz - 1)) : 0;
    const int na = axis == 0 ? dy : dx;
    const int nb = axis == 2 ? dy : dz;
    float m = 3.0e38f;
    for (int t = threadIdx.x; t < na * nb; t += blockDim.x) {
        const int a = t / nb, b = t % nb;
        int x, y, z;
        if (axis == 0) { x = fixed; y = a; z = b; }
        else if (axis == 1) { x = a; y = fixed; z = b; }
        else { x = a; y = b; z = fixed; }
        m = fminf(m, dist[((long)x * dy + y) * dz + z]);
    }
    __shared__ float sm[32];
    for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < (blockDim.x >> 5) ? sm[threadIdx.x] : 3.0e38f;
        for (int o = 16; o > 0; o >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) out[face] = m;
    }
}

void launch_sdf_slab_min(const float* dist, int dx, int dy, int dz, float* slab_min, cudaStream_t st)
{
    k_sdf_slab_min<<<6, 256, 0, st>>>(dist, dx, dy, dz, slab_min);
}

__global__ void k_sdf_sample(SdfDev S, const float* __restrict__ pts, uint32_t n, float* __restrict__ d,
                             float* __restrict__ grad)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
    d[i] = sdf_sample(S, x, y, z);
    if (grad) {
        const float e = S.cell;
        const float inv2e = 1.0f / (2.0f * e);
        grad[3 * i] = (sdf_sample(S, x + e, y, z) - sdf_sample(S, x - e, y, z)) * inv2e;
        grad[3 * i + 1] = (sdf_sample(S, x, y + e, z) - sdf_sample(S, x, y - e, z)) * inv2e;
        grad[3 * i + 2] = (sdf_sample(S, x, y, z + e) - sdf_sample(S, x, y, z - e)) * inv2e;
    }
}

void launch_sdf_sample(SdfDev S, const float* pts3, uint32_t n, float* d, float* grad3, cudaStream_t st)
{
    if (n == 0) return;
    k_sdf_sample<<<(n + 255) / 256, 256, 0, st>>>(S, pts3, n, d, grad3);
}

// ---- contact compaction (CS_ContactFilter.glsl:68-83, deterministic) --------
constexpr int kCtThreads = 256;
constexpr int kCtItems = 4;
constexpr int kCtBlock = kCtThreads * kCtItems;

uint32_t contact_num_blocks(uint32_t n) { return (n + kCtBlock - 1) / kCtBlock; }

__device__ __forceinline__ bool in_band(const SdfDev& S, float4 p, float band)
{
    return fabsf(sdf_sample(S, p.x, p.y, p.z)) < band;
}

__global__ void __launch_bounds__(kCtThreads) k_contact_count(SdfDev S, uint32_t n, const float4* __restrict__ pos,
                                                              float band, uint32_t* __restrict__ counts)
{
    uint32_t c = 0;
    const uint32_t base = blockIdx.x * kCtBlock;
#pragma unroll
    for (int r = 0; r < kCtItems; ++r) {
        const uint32_t i = base + r * kCtThreads + threadIdx.x;
        if (i < n && in_band(S, __ldg(pos + i), band)) ++c;
    }
    __shared__ uint32_t sm[kCtThreads / 32];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kCtThreads / 32; ++w) t += sm[w];
        counts[blockIdx.x] = t;
    }
}

// exclusive scan of the block counts in one block; total to *total
__global__ void __launch_bounds__(1024) k_contact_scan(uint32_t* __restrict__ counts, uint32_t nb,
                                                       uint32_t* __restrict__ total)
{
    __shared__ uint32_t ws[32];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < nb; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nb ? counts[i] : 0u;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
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
        const uint32_t ex = carry + incl - v + (warp ? ws[warp - 1] : 0u);
        if (i < nb) counts[i] = ex;
        const uint32_t chunk_total = ws[31];
        __syncthreads();
        carry += chunk_total;
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kCtThreads) k_contact_write(SdfDev S, uint32_t n, const float4* __restrict__ pos,
                                                              const float4* __restrict__ vel, float band,
                                                              const uint32_t* __restrict__ offsets,
                                                              float4* __restrict__ out)
{
    __shared__ uint32_t ws[kCtThreads / 32];
    const uint32_t base = blockIdx.x * kCtBlock;
    uint32_t run = offsets[blockIdx.x];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = 0; r < kCtItems; ++r) {
        const uint32_t i = base + r * kCtThreads + threadIdx.x;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        bool f = false;
        if (i < n) {
            p = __ldg(pos + i);
            f = in_band(S, p, band);
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) ws[warp] = __popc(bal);
        __syncthreads();
        uint32_t woff = 0, all = 0;
        for (int w = 0; w < kCtThreads / 32; ++w) {
            if (w < warp) woff += ws[w];
            all += ws[w];
        }
        if (f) {
            const uint32_t slot = run + woff + __popc(bal & ((1u << lane) - 1u));
            out[2 * slot] = make_float4(p.x, p.y, p.z, 0.0f);  // vec4(pos, 0.0)
            out[2 * slot + 1] = __ldg(vel + i);                 // particles[id].vel (w = pad)
        }
        run += all;
        __syncthreads();
    }
}

void launch_contact_filter(SdfDev S, uint32_t n, const float4* pos, const float4* vel, float band,
                           uint32_t* block_counts, uint32_t* total, float4* out_cand, cudaStream_t st,
                           uint64_t* launches)
{
    const uint32_t nb = contact_num_blocks(n);
    k_contact_count<<<nb, kCtThreads, 0, st>>>(S, n, pos, band, block_counts);
    k_contact_scan<<<1, 1024, 0, st>>>(block_counts, nb, total);
    k_contact_write<<<nb, kCtThreads, 0, st>>>(S, n, pos, vel, band, block_counts, out_cand);
    if (launches) *launches += 3;
}

}  // namespace pbf
