/*
 * sdf_ref_bridge.cpp — C entry points over the reference's own
 * SDFBoundary (src/fluid/SDFBoundary.cpp, compiled as it lies in the
 * reference tree with the shims of oracle/shim).  TEST INFRASTRUCTURE ONLY:
 * built into oracle/_ref/libpbfref_sdf.so and used by tests/ to pin the mesh
 * half of the oracle and the GPU mesh kernels to the reference.
 */
#include <array>
#include <vector>

#include "fluid/SDFBoundary.h"

namespace {
std::vector<std::array<double, 3>> verts_of(const double* v3, int nv)
{
    std::vector<std::array<double, 3>> v((size_t)nv);
    for (int i = 0; i < nv; ++i) v[(size_t)i] = {v3[3 * i], v3[3 * i + 1], v3[3 * i + 2]};
    return v;
}
}  // namespace

extern "C" {

void* sdfref_build(const double* verts3, int nv, const int* faces3, int nf, double resolution)
{
    std::vector<std::array<int, 3>> f((size_t)nf);
    for (int i = 0; i < nf; ++i) f[(size_t)i] = {faces3[3 * i], faces3[3 * i + 1], faces3[3 * i + 2]};
    SDFBoundary* s = new SDFBoundary();
    s->buildFromMesh(verts_of(verts3, nv), f, resolution, false);
    return s;
}

void sdfref_free(void* h) { delete static_cast<SDFBoundary*>(h); }

void sdfref_grid_info(void* h, int* dims3, double* origin3, double* cell)
{
    const SDFBoundary* s = static_cast<const SDFBoundary*>(h);
    dims3[0] = s->dimensions().x();
    dims3[1] = s->dimensions().y();
    dims3[2] = s->dimensions().z();
    origin3[0] = s->origin().x();
    origin3[1] = s->origin().y();
    origin3[2] = s->origin().z();
    *cell = s->cellSize();
}

/* CPU grid order: index = x*dy*dz + y*dz + z */
void sdfref_grid(void* h, float* out)
{
    const std::vector<float>& d = static_cast<const SDFBoundary*>(h)->distances();
    for (size_t i = 0; i < d.size(); ++i) out[i] = d[i];
}

void sdfref_refit(void* h, const double* verts3, int nv) { static_cast<SDFBoundary*>(h)->refitFromMesh(verts_of(verts3, nv)); }

int sdfref_refit_dirty(void* h, const double* verts3, int nv, double band, double move_eps)
{
    return static_cast<SDFBoundary*>(h)->refitDirty(verts_of(verts3, nv), band, move_eps) ? 1 : 0;
}

void sdfref_closest(void* h, const float* pts3, int n, int* face, float* point3)
{
    const SDFBoundary* s = static_cast<const SDFBoundary*>(h);
    for (int i = 0; i < n; ++i) {
        const SDFBoundary::ClosestSurface c = s->closestTriangle(PVec3{pts3[3 * i], pts3[3 * i + 1], pts3[3 * i + 2]});
        face[i] = c.face;
        point3[3 * i] = c.point.x;
        point3[3 * i + 1] = c.point.y;
        point3[3 * i + 2] = c.point.z;
    }
}

}  // extern "C"
