// fluid/SDFBoundary.h — signed-distance boundary for fluid-solid coupling.
//
// Drop-in for the reference's include/fluid/SDFBoundary.h:38-167.  The build,
// refit, grid and closest-triangle queries run on the GPU (LBVH over the
// faces, grid recomputed from it); `uploadToGPU`, `uploadDirtyRegion` and
// `bindForQuery` are no-ops kept for source compatibility.  origin() and
// dimensions() return small value types with the x()/y()/z() accessors the
// reference's Eigen return types offer.
#ifndef PBF_B200_FLUID_SDFBOUNDARY_H
#define PBF_B200_FLUID_SDFBOUNDARY_H

#include <array>
#include <vector>

#include "core/Types.h"

struct pbf_handle;

namespace pbfdrop {
struct Vec3d {
    double v[3] = {0, 0, 0};
    double x() const { return v[0]; }
    double y() const { return v[1]; }
    double z() const { return v[2]; }
    double operator[](int i) const { return v[i]; }
};
struct Vec3i {
    int v[3] = {0, 0, 0};
    int x() const { return v[0]; }
    int y() const { return v[1]; }
    int z() const { return v[2]; }
    int operator[](int i) const { return v[i]; }
};
}  // namespace pbfdrop

class SDFBoundary {
public:
    SDFBoundary();
    explicit SDFBoundary(int device);
    ~SDFBoundary();
    SDFBoundary(const SDFBoundary&) = delete;
    SDFBoundary& operator=(const SDFBoundary&) = delete;

    // A build of the same faces at the same resolution as the last one (the
    // reference's periodic rebuild of a deforming mesh, main.cpp:326) runs
    // entirely on the GPU: LBVH, face, edge and vertex pseudo-normals, grid.
    void buildFromMesh(const std::vector<std::array<double, 3>>& verts, const std::vector<std::array<int, 3>>& faces,
                       double resolution, bool verbose = true);
    void refitFromMesh(const std::vector<std::array<double, 3>>& verts);
    bool refitDirty(const std::vector<std::array<double, 3>>& newVerts, double bandRadius, double moveEps);
    void setDebugVerifyDirty(bool on) { _debugVerifyDirty = on; }

    void uploadToGPU() {}
    void uploadDirtyRegion() {}
    void bindForQuery(unsigned int /*textureUnit*/) const {}

    bool valid() const { return _valid; }
    const pbfdrop::Vec3d& origin() const { return _origin; }
    double cellSize() const { return _cellSize; }
    const pbfdrop::Vec3i& dimensions() const { return _dimensions; }
    // Host copy of the grid (read back from the GPU on first use after a change).
    const std::vector<float>& distances() const;
    int index(int x, int y, int z) const { return x * _dimensions.y() * _dimensions.z() + y * _dimensions.z() + z; }

    struct ClosestSurface {
        int face = -1;
        PVec3 point{0.f, 0.f, 0.f};
    };
    ClosestSurface closestTriangle(const PVec3& p) const;

    // engine handle holding the GPU field (used by PBFluids::setSDFBoundary)
    pbf_handle* handle() const { return _h; }

private:
    void refreshInfo();
    pbf_handle* _h = nullptr;
    bool _valid = false;
    bool _debugVerifyDirty = false;
    pbfdrop::Vec3d _origin;
    double _cellSize = 0.0;
    pbfdrop::Vec3i _dimensions;
    std::vector<std::array<double, 3>> _buildVerts;
    std::vector<std::array<int, 3>> _buildFaces;
    double _buildResolution = 0.0;
    mutable std::vector<float> _distances;
    mutable bool _distancesStale = true;
};

#endif
