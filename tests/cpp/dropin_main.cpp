// Drop-in check: a caller written against the reference's fluid interface
// (the construct -> setParams -> setParticles -> SDF -> step -> contacts ->
// refit sequence of the reference's src/main.cpp:446-497, 959-990, 1673-1708)
// compiled against include/fluid/*.h and linked with libpbf_b200.so.
#include <array>
#include <cmath>
#include <cstdio>
#include <vector>

#include "core/Config.h"
#include "fluid/PBFluids.h"
#include "fluid/SDFBoundary.h"

static void octahedron_sphere(double r, const double c[3], std::vector<std::array<double, 3>>& V,
                              std::vector<std::array<int, 3>>& F, int rings = 24, int segs = 48)
{
    // UV sphere, outward-oriented faces
    V.clear();
    F.clear();
    V.push_back({c[0], c[1] + r, c[2]});
    for (int i = 1; i < rings; ++i) {
        const double th = M_PI * i / rings;
        for (int j = 0; j < segs; ++j) {
            const double ph = 2 * M_PI * j / segs;
            V.push_back({c[0] + r * std::sin(th) * std::cos(ph), c[1] + r * std::cos(th), c[2] + r * std::sin(th) * std::sin(ph)});
        }
    }
    V.push_back({c[0], c[1] - r, c[2]});
    const int bottom = (int)V.size() - 1;
    for (int j = 0; j < segs; ++j) F.push_back({0, 1 + (j + 1) % segs, 1 + j});
    for (int i = 0; i < rings - 2; ++i)
        for (int j = 0; j < segs; ++j) {
            const int a = 1 + i * segs + j, b = 1 + i * segs + (j + 1) % segs;
            const int cc = a + segs, d = b + segs;
            F.push_back({a, b, d});
            F.push_back({a, d, cc});
        }
    const int base = 1 + (rings - 2) * segs;
    for (int j = 0; j < segs; ++j) F.push_back({bottom, base + j, base + (j + 1) % segs});
}

int main()
{
    Config cfg;
    FluidConfig& fc = cfg.fluid;
    fc.h = 0.04f;
    fc.spacing = 0.02f;
    fc.rho0 = 126221.896f;
    fc.eps = 100.0f;
    fc.kCorr = 0.1f;
    fc.deltaQ = 0.2f;
    fc.viscosity = 0.01f;
    fc.vorticityEpsilon = 0.0005f;
    fc.gravity = {0.f, -9.81f, 0.f};
    fc.solverIterations = 4;
    fc.substepIterations = 2;
    fc.boundsMin = {0.f, 0.f, 0.f};
    fc.boundsMax = {1.6f, 1.0f, 1.0f};

    PBFluids fluid(fc);
    fluid.setCollisionPadding(0.0f);
    fluid.setParams(fc);
    fluid.setBounds(fc.boundsMin, fc.boundsMax, fc.boundDamping);

    std::vector<Particle> ps;
    for (int z = 0; z < 16; ++z)
        for (int y = 0; y < 16; ++y)
            for (int x = 0; x < 16; ++x) {
                Particle p{};
                p.pos = {0.6f + (x + 0.5f) * 0.02f, 0.45f + (y + 0.5f) * 0.02f, 0.34f + (z + 0.5f) * 0.02f};
                p.predPos = p.pos;
                ps.push_back(p);
            }
    fluid.setParticles(ps);

    SDFBoundary sdf;
    std::vector<std::array<double, 3>> V;
    std::vector<std::array<int, 3>> F;
    const double center[3] = {0.76, 0.2, 0.5};
    octahedron_sphere(0.15, center, V, F);
    sdf.buildFromMesh(V, F, 0.02, false);
    sdf.uploadToGPU();
    fluid.setSDFBoundary(&sdf);
    fluid.setSDFPadding(0.01f);
    fluid.setSDFContainment(false);

    std::vector<ContactCandidate> cand;
    std::vector<PVec3> forces(V.size());
    int total_contacts = 0;
    for (int frame = 0; frame < 40; ++frame) {
        fluid.readbackContactCandidates(cand);
        total_contacts += fluid.computeContactForces(0.06f, true, forces);
        // a small dent following the push, then the refresh the reference does
        for (size_t i = 0; i < V.size(); ++i) {
            V[i][0] += 1e-4 * forces[i].x;
            V[i][1] += 1e-4 * forces[i].y;
            V[i][2] += 1e-4 * forces[i].z;
        }
        sdf.refitDirty(V, 0.05, 1e-4);
        fluid.setSDFBoundary(&sdf);
        fluid.step();
        fluid.filterContactCandidates(0.06f);
    }
    std::vector<Particle> out;
    fluid.readbackParticles(out);
    int bad = 0, inside = 0;
    for (const Particle& p : out) {
        if (!std::isfinite(p.pos.x) || !std::isfinite(p.vel.y)) ++bad;
        const double dx = p.pos.x - center[0], dy = p.pos.y - center[1], dz = p.pos.z - center[2];
        if (std::sqrt(dx * dx + dy * dy + dz * dz) < 0.15 - 0.01) ++inside;
    }
    const auto d = sdf.dimensions();
    const auto closest = sdf.closestTriangle(PVec3{0.76f, 0.5f, 0.5f});
    std::printf("{\"particles\": %zu, \"nonfinite\": %d, \"inside_obstacle\": %d, \"contacts\": %d, "
                "\"grid\": [%d, %d, %d], \"closest_face\": %d, \"grid_voxels_read\": %zu}\n",
                out.size(), bad, inside, total_contacts, d.x(), d.y(), d.z(), closest.face, sdf.distances().size());
    return (bad == 0 && inside == 0 && out.size() == ps.size() && total_contacts > 0 && closest.face >= 0) ? 0 : 1;
}
