// k_masked.cu — neighbour passes that test a bucket chunk first and run the
// in-range body only for the hits (thread per particle, Morton order).
//
// A warp runs the pair body as many times per bucket as its busiest lane has
// hits (about 3 at h/d = 2) instead of once per candidate step on which any
// lane has a hit, and the 8 loads of a chunk are in flight together.  The
// per-particle bodies live in masked_body.cuh.
#include "masked_body.cuh"
#include "pbf_kernels.h"

namespace pbf {

constexpr int kMThreads = 128;

__global__ void __launch_bounds__(kMThreads) k_lambda_m(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, float* __restrict__ rho_out,
                                                        const int2* __restrict__ table, const uint32_t* __restrict__ lod,
                                                        uint32_t iter, const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    if (P.apbf && __ldg(lod + s) < iter) {
        xout[s] = __ldg(xin + s);
        return;
    }
    float rho;
    xout[s] = lambda_particle(P, table, P.mask, xin, s, rho);
    rho_out[s] = rho;
}

__global__ void __launch_bounds__(kMThreads) k_deltap_m(DevParams P, const float4* __restrict__ xin,
                                                        float4* __restrict__ xout, const int2* __restrict__ table,
                                                        const uint32_t* __restrict__ lod, uint32_t iter,
                                                        const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    if (P.apbf && __ldg(lod + s) < iter) {
        xout[s] = __ldg(xin + s);
        return;
    }
    xout[s] = deltap_particle(P, table, P.mask, P.sdf, xin, s);
}

__global__ void __launch_bounds__(kMThreads) k_integrate_m(DevParams P, const float4* __restrict__ xs,
                                                           const float4* __restrict__ sv, float4* __restrict__ sx0,
                                                           float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ pos,
                                                           float4* __restrict__ vel, const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    integrate_particle(P, table, P.mask, P.bmin, P.bmax, P.sdf, xs, sv, sx0, somega, ids, pos, vel, s);
}

__global__ void __launch_bounds__(kMThreads) k_vorticity_m(DevParams P, const float4* __restrict__ spos,
                                                           const float4* __restrict__ somega,
                                                           const uint32_t* __restrict__ ids, float4* __restrict__ vel,
                                                           const int2* __restrict__ table,
                                                           const uint32_t* __restrict__ order)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int)P.n) return;
    const int s = order ? (int)__ldg(order + t) : t;
    vorticity_particle(P, table, P.mask, spos, somega, ids, vel, s);
}

static inline unsigned mgrid(uint32_t n) { return (n + kMThreads - 1) / kMThreads; }

void launch_lambda_m(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                     const uint32_t* lod, uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    k_lambda_m<<<mgrid(P.n), kMThreads, 0, st>>>(P, xin, xout, rho, table, lod, iter, order);
}

void launch_deltap_m(const DevParams& P, const float4* xin, float4* xout, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, cudaStream_t st)
{
    k_deltap_m<<<mgrid(P.n), kMThreads, 0, st>>>(P, xin, xout, table, lod, iter, order);
}

void launch_integrate_m(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                        const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                        cudaStream_t st)
{
    k_integrate_m<<<mgrid(P.n), kMThreads, 0, st>>>(P, xs, sv, sx0, somega, ids, pos, vel, table, order);
}

void launch_vorticity_m(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                        float4* vel, const int2* table, const uint32_t* order, cudaStream_t st)
{
    k_vorticity_m<<<mgrid(P.n), kMThreads, 0, st>>>(P, spos, somega, ids, vel, table, order);
}

}  // namespace pbf
