// ref_bridge.cpp — extern "C" entry points over the reference's own CPU
// code (src/fluid/Kernels.cpp, src/fluid/NeighborSearch.cpp), compiled from
// the reference tree into oracle/_ref/libpbfref_cpu.so by oracle/Makefile.
//
// TEST INFRASTRUCTURE ONLY: used to pin the FP64 oracle (golden vectors in
// tests/golden) and as a reference-code CPU baseline.
#include <cstdint>
#include <cstring>
#include <vector>

#include "core/Types.h"
#include "fluid/Kernels.h"
#include "fluid/NeighborSearch.h"
#include "fluid/Particle.h"

extern "C" {

float ref_poly6(float rx, float ry, float rz, float h) { return calcPoly6Kernel(make_pvec3(rx, ry, rz), h); }

void ref_grad_spiky(float rx, float ry, float rz, float h, float* out3)
{
    const PVec3 g = calcGradSpikyPow3Kernel(make_pvec3(rx, ry, rz), h);
    out3[0] = g.x;
    out3[1] = g.y;
    out3[2] = g.z;
}

float ref_scorr_kernel(float rx, float ry, float rz, float h) { return calcSCorrKernel(make_pvec3(rx, ry, rz), h); }

// NeighborSearch::build over particles whose predPos = pred3[i]; writes the
// per-particle neighbour count and, when `lists` is non-null, up to
// `cap_per_particle` neighbour ids per particle.  Returns the total number
// of neighbour entries.
int64_t ref_neighbor_build(const float* pred3, int32_t n, float cell, uint32_t hash_size,
                           int32_t* counts, int32_t* lists, int32_t cap_per_particle)
{
    std::vector<Particle> ps(static_cast<size_t>(n));
    for (int32_t i = 0; i < n; ++i) {
        ps[i].predPos = make_pvec3(pred3[3 * i], pred3[3 * i + 1], pred3[3 * i + 2]);
        ps[i].pos = ps[i].predPos;
    }
    NeighborSearch ns(cell, hash_size);
    ns.build(ps);
    int64_t total = 0;
    for (int32_t i = 0; i < n; ++i) {
        const std::vector<I32>& nb = ns.getNeighbors(i);
        counts[i] = static_cast<int32_t>(nb.size());
        if (lists) {
            const int32_t m = static_cast<int32_t>(nb.size()) < cap_per_particle ? static_cast<int32_t>(nb.size())
                                                                                   : cap_per_particle;
            for (int32_t k = 0; k < m; ++k) lists[static_cast<int64_t>(i) * cap_per_particle + k] = nb[k];
        }
        total += static_cast<int64_t>(nb.size());
    }
    return total;
}

}  // extern "C"
