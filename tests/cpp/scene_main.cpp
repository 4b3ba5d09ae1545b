// Headless scene check: the reference's preset 0 ("Container Cube",
// include/core/Scene.h) set up through include/core/SceneSetup.h's loadScene
// exactly as a C++ caller would, with a cube of the asset's topology (a
// 16 x 16 grid per face) written here as an OFF file in place of the
// reference's cube1538.off.  Steps 30 frames and prints one JSON line:
// particle count, non-finite values, particles outside the cube.
#include <array>
#include <cmath>
#include <cstdio>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "core/Scene.h"
#include "core/SceneSetup.h"
#include "fluid/PBFluids.h"
#include "fluid/SDFBoundary.h"

static bool write_grid_cube(const std::string& path, int n)
{
    std::map<std::tuple<int, int, int>, int> index;
    std::vector<std::array<double, 3>> V;
    std::vector<std::array<int, 3>> F;
    auto vid = [&](int a, int b, int c) {
        const auto key = std::make_tuple(a, b, c);
        auto it = index.find(key);
        if (it != index.end()) return it->second;
        const int id = (int)V.size();
        V.push_back({-0.5 + (double)a / n, -0.5 + (double)b / n, -0.5 + (double)c / n});
        index[key] = id;
        return id;
    };
    for (int axis = 0; axis < 3; ++axis)
        for (int side = 0; side < 2; ++side)
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) {
                    int q[4];
                    const int du[4] = {0, 1, 1, 0}, dv[4] = {0, 0, 1, 1};
                    for (int k = 0; k < 4; ++k) {
                        int c[3];
                        c[axis] = side * n;
                        c[(axis + 1) % 3] = i + du[k];
                        c[(axis + 2) % 3] = j + dv[k];
                        q[k] = vid(c[0], c[1], c[2]);
                    }
                    if (side) {
                        F.push_back({q[0], q[1], q[2]});
                        F.push_back({q[0], q[2], q[3]});
                    } else {
                        F.push_back({q[0], q[2], q[1]});
                        F.push_back({q[0], q[3], q[2]});
                    }
                }
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "OFF\n%zu %zu 0\n", V.size(), F.size());
    for (const auto& v : V) std::fprintf(f, "%.9g %.9g %.9g\n", v[0], v[1], v[2]);
    for (const auto& t : F) std::fprintf(f, "3 %d %d %d\n", t[0], t[1], t[2]);
    std::fclose(f);
    return true;
}

int main(int argc, char** argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    if (!write_grid_cube(dir + "/cube1538.off", 16)) return 2;
    const Scene& sc = getScenes()[0];
    PBFluids fluid;
    SDFBoundary sdf;
    SceneState st;
    if (!loadScene(sc, dir, fluid, sdf, &st)) return 3;
    for (int f = 0; f < 30; ++f) fluid.step();
    std::vector<Particle> out;
    fluid.readbackParticles(out);
    int nonfinite = 0, outside = 0;
    // the fitted, placed cube: centre of the walls in x and z, 40 % up plus
    // the preset's 0.5 lift in y, edge meshFitSize
    const PVec3 c = meshFitCenter(sc.fluid);
    const float half = 0.5f * sc.meshFitSize;
    for (const Particle& p : out) {
        if (!std::isfinite(p.pos.x) || !std::isfinite(p.pos.y) || !std::isfinite(p.pos.z)) ++nonfinite;
        const float dx = std::fabs(p.pos.x - c.x), dy = std::fabs(p.pos.y - (c.y + sc.meshTranslate.y)),
                    dz = std::fabs(p.pos.z - c.z);
        if (dx > half || dy > half || dz > half) ++outside;
    }
    std::printf("{\"particles\": %zu, \"mesh_vertices\": %zu, \"mesh_faces\": %zu, \"nonfinite\": %d, \"outside\": %d}\n",
                out.size(), st.mesh.verts.size(), st.mesh.faces.size(), nonfinite, outside);
    return 0;
}
