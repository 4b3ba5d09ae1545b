// harness.cpp — runs the reference's compute shaders (translated to C++ by
// oracle/glsl/translate.py) on the CPU, dispatch by dispatch, in the order
// PBFluids::step issues them (src/fluid/PBFluids.cpp:323-517).
//
// TEST INFRASTRUCTURE ONLY.  Built into oracle/_ref/libpbfref_glsl.so.
// Barrier-free shaders run one invocation per loop iteration (optionally
// OpenMP-parallel); the radix-sort shaders, which use shared memory and
// barrier(), run each workgroup as 256 threads meeting at a std::barrier.
#include <algorithm>
#include <barrier>
#include <cstring>
#include <thread>
#include <vector>

#include "glsl_shim.hpp"

namespace glsl {
static thread_local std::barrier<>* t_wg_barrier = nullptr;
inline void barrier() { t_wg_barrier->arrive_and_wait(); }
}  // namespace glsl

#include "cs_ApplyDeltaP.inc"
#include "cs_BuildOffsets.inc"
#include "cs_ComputeDeltaP.inc"
#include "cs_ComputeLOD.inc"
#include "cs_ComputeLambdas.inc"
#include "cs_ContactFilter.inc"
#include "cs_Integrate.inc"
#include "cs_PredictAndHash.inc"
#include "cs_RadixHistogram.inc"
#include "cs_RadixPrefixSum.inc"
#include "cs_RadixScatter.inc"
#include "cs_VorticityConfinement.inc"
#include "harness.h"

using namespace glsl;

namespace {

template <class Body>
void dispatch(uint32_t groups, bool parallel, Body body)
{
    const long total = (long)groups * 256;
    if (parallel) {
#pragma omp parallel for schedule(static)
        for (long g = 0; g < total; ++g) body((uint)g);
    } else {
        for (long g = 0; g < total; ++g) body((uint)g);
    }
}

template <class Body>
void dispatch_workgroups(uint32_t groups, Body body)
{
    for (uint32_t g = 0; g < groups; ++g) {
        std::barrier<> bar(256);
        std::vector<std::thread> th;
        th.reserve(256);
        for (uint32_t l = 0; l < 256; ++l)
            th.emplace_back([&bar, &body, g, l] {
                t_wg_barrier = &bar;
                body(g, l);
            });
        for (auto& t : th) t.join();
    }
}

template <class UBO>
void set_ubo(UBO& dst, const pbf_derived_params& src)
{
    static_assert(sizeof(UBO) <= sizeof(pbf_derived_params), "UBO prefix");
    std::memcpy(&dst, &src, sizeof(UBO));
}

std::vector<float> g_tex;  // SDF in GL texture order (x fastest)

sampler3D make_sampler(const glsl_ref_ctx* c)
{
    sampler3D s;
    if (!c->enable_sdf || !c->sdf_dist) return s;
    const int W = c->sdf_dims[0], H = c->sdf_dims[1], D = c->sdf_dims[2];
    g_tex.assign((size_t)W * H * D, 0.0f);
    // uploadToGPU repack (SDFBoundary.cpp:587-595)
    for (int z = 0; z < D; ++z)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x)
                g_tex[(size_t)x + (size_t)W * ((size_t)y + (size_t)H * z)] = c->sdf_dist[((size_t)x * H + y) * D + z];
    s.texels = g_tex.data();
    s.w = W;
    s.h = H;
    s.d = D;
    return s;
}

void radix_sort(glsl_ref_ctx* c)
{
    const uint32_t N = c->n;
    const uint32_t groups = (N + 255u) / 256u;
    if (c->sort_mode == 0) {
        // The shader chain below is a stable LSD sort on the key column.
        std::vector<std::pair<uint32_t, uint32_t>> v(N);
        for (uint32_t i = 0; i < N; ++i) v[i] = {c->hash_grid[2 * i], c->hash_grid[2 * i + 1]};
        std::stable_sort(v.begin(), v.end(), [](auto& a, auto& b) { return a.first < b.first; });
        for (uint32_t i = 0; i < N; ++i) {
            c->hash_grid[2 * i] = v[i].first;
            c->hash_grid[2 * i + 1] = v[i].second;
        }
        return;
    }
    // PBFluids.cpp:354-405: 4 passes of histogram / prefix sum / scatter.
    bool source_is_primary = true;
    for (uint32_t pass = 0; pass < 4; ++pass) {
        uvec2* src = (uvec2*)(source_is_primary ? c->hash_grid : c->hash_grid_alt);
        uvec2* dst = (uvec2*)(source_is_primary ? c->hash_grid_alt : c->hash_grid);
        cs_RadixHistogram::source = src;
        cs_RadixHistogram::histogram = c->histogram;
        cs_RadixHistogram::bitOffset = pass * 8;
        cs_RadixHistogram::particleCount = N;
        cs_RadixHistogram::numWorkgroups = groups;
        dispatch_workgroups(groups, [](uint32_t g, uint32_t l) {
            cs_RadixHistogram::gl_WorkGroupID = uvec3{g, 0, 0};
            cs_RadixHistogram::gl_LocalInvocationID = uvec3{l, 0, 0};
            cs_RadixHistogram::gl_GlobalInvocationID = uvec3{g * 256 + l, 0, 0};
            cs_RadixHistogram::main();
        });
        cs_RadixPrefixSum::histogram = c->histogram;
        cs_RadixPrefixSum::totalCount = groups * 256;
        dispatch_workgroups(1, [](uint32_t g, uint32_t l) {
            cs_RadixPrefixSum::gl_WorkGroupID = uvec3{g, 0, 0};
            cs_RadixPrefixSum::gl_LocalInvocationID = uvec3{l, 0, 0};
            cs_RadixPrefixSum::gl_GlobalInvocationID = uvec3{g * 256 + l, 0, 0};
            cs_RadixPrefixSum::main();
        });
        cs_RadixScatter::source = src;
        cs_RadixScatter::dest = dst;
        cs_RadixScatter::histogram = c->histogram;
        cs_RadixScatter::bitOffset = pass * 8;
        cs_RadixScatter::particleCount = N;
        cs_RadixScatter::numWorkgroups = groups;
        dispatch_workgroups(groups, [](uint32_t g, uint32_t l) {
            cs_RadixScatter::gl_WorkGroupID = uvec3{g, 0, 0};
            cs_RadixScatter::gl_LocalInvocationID = uvec3{l, 0, 0};
            cs_RadixScatter::gl_GlobalInvocationID = uvec3{g * 256 + l, 0, 0};
            cs_RadixScatter::main();
        });
        source_is_primary = !source_is_primary;
    }
}

void bind_all(glsl_ref_ctx* c)
{
    set_ubo(cs_PredictAndHash::ubo, c->ubo);
    set_ubo(cs_BuildOffsets::ubo, c->ubo);
    set_ubo(cs_ComputeLOD::ubo, c->ubo);
    set_ubo(cs_ComputeLambdas::ubo, c->ubo);
    set_ubo(cs_ComputeDeltaP::ubo, c->ubo);
    set_ubo(cs_ApplyDeltaP::ubo, c->ubo);
    set_ubo(cs_Integrate::ubo, c->ubo);
    set_ubo(cs_VorticityConfinement::ubo, c->ubo);
    set_ubo(cs_ContactFilter::ubo, c->ubo);

    cs_PredictAndHash::particles = (cs_PredictAndHash::Particle*)c->particles;
    cs_PredictAndHash::solver = (cs_PredictAndHash::SolverData*)c->solver;
    cs_PredictAndHash::hashGrid = (uvec2*)c->hash_grid;
    cs_PredictAndHash::isInteracting = c->is_interacting;
    cs_PredictAndHash::interactionPos = make_vec3(c->interaction_pos[0], c->interaction_pos[1], c->interaction_pos[2]);

    cs_BuildOffsets::hashGrid = (uvec2*)c->hash_grid;
    cs_BuildOffsets::offsets = (ivec2*)c->offsets;

    cs_ComputeLOD::solver = (cs_ComputeLOD::SolverData*)c->solver;
    cs_ComputeLOD::lod = c->lod;
    cs_ComputeLOD::cameraPos = make_vec3(c->camera_pos[0], c->camera_pos[1], c->camera_pos[2]);

    cs_ComputeLambdas::solver = (cs_ComputeLambdas::SolverData*)c->solver;
    cs_ComputeLambdas::hashGrid = (uvec2*)c->hash_grid;
    cs_ComputeLambdas::offsets = (ivec2*)c->offsets;
    cs_ComputeLambdas::lod = c->lod;

    cs_ComputeDeltaP::solver = (cs_ComputeDeltaP::SolverData*)c->solver;
    cs_ComputeDeltaP::hashGrid = (uvec2*)c->hash_grid;
    cs_ComputeDeltaP::offsets = (ivec2*)c->offsets;
    cs_ComputeDeltaP::lod = c->lod;

    const sampler3D tex = make_sampler(c);
    const vec4 org = make_vec4(c->sdf_origin[0], c->sdf_origin[1], c->sdf_origin[2], 0.0f);
    const vec4 res = make_vec4((float)c->sdf_dims[0], (float)c->sdf_dims[1], (float)c->sdf_dims[2], 0.0f);
    const uint sdf_on = (c->enable_sdf && c->sdf_dist) ? 1u : 0u;

    cs_ApplyDeltaP::solver = (cs_ApplyDeltaP::SolverData*)c->solver;
    cs_ApplyDeltaP::lod = c->lod;
    cs_ApplyDeltaP::enableSDF = sdf_on;
    cs_ApplyDeltaP::sdfMode = c->sdf_mode;
    cs_ApplyDeltaP::sdfTexture = tex;
    cs_ApplyDeltaP::sdfOrigin = org;
    cs_ApplyDeltaP::sdfCellSize = c->sdf_cell;
    cs_ApplyDeltaP::sdfResolution = res;
    cs_ApplyDeltaP::sdfPadding = c->sdf_padding;

    cs_Integrate::particles = (cs_Integrate::Particle*)c->particles;
    cs_Integrate::particles_prev = (cs_Integrate::Particle*)c->particles;
    cs_Integrate::solver = (cs_Integrate::SolverData*)c->solver;
    cs_Integrate::hashGrid = (uvec2*)c->hash_grid;
    cs_Integrate::offsets = (ivec2*)c->offsets;
    cs_Integrate::enableVorticity = c->enable_vorticity;
    cs_Integrate::enableSDF = sdf_on;
    cs_Integrate::sdfMode = c->sdf_mode;
    cs_Integrate::sdfTexture = tex;
    cs_Integrate::sdfOrigin = org;
    cs_Integrate::sdfCellSize = c->sdf_cell;
    cs_Integrate::sdfResolution = res;
    cs_Integrate::sdfPadding = c->sdf_padding;

    cs_VorticityConfinement::particles = (cs_VorticityConfinement::Particle*)c->particles;
    cs_VorticityConfinement::solver = (cs_VorticityConfinement::SolverData*)c->solver;
    cs_VorticityConfinement::hashGrid = (uvec2*)c->hash_grid;
    cs_VorticityConfinement::offsets = (ivec2*)c->offsets;
    cs_VorticityConfinement::vorticityEpsilon = c->vorticity_epsilon;
    cs_VorticityConfinement::pass = 1u;

    cs_ContactFilter::particles = (cs_ContactFilter::Particle*)c->particles;
    cs_ContactFilter::contactCount__p = c->contact_count;
    cs_ContactFilter::candidates = (cs_ContactFilter::ContactCandidate*)c->contacts;
    cs_ContactFilter::sdfTexture = tex;
    cs_ContactFilter::sdfOrigin = org;
    cs_ContactFilter::sdfCellSize = c->sdf_cell;
    cs_ContactFilter::sdfResolution = res;
    cs_ContactFilter::contactBand = c->contact_band;
}

int run_stage(glsl_ref_ctx* c, int stage, uint32_t iter)
{
    const uint32_t N = c->n;
    const uint32_t groups = (N + 255u) / 256u;
    const uint32_t grid_groups = (c->ubo.hash_size + 255u) / 256u;
    const bool par = c->parallel != 0;
    switch (stage) {
    case GLSL_PREDICT:
        dispatch(groups, par, [](uint g) {
            cs_PredictAndHash::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_PredictAndHash::main();
        });
        return 0;
    case GLSL_SORT:
        radix_sort(c);
        return 0;
    case GLSL_OFFSETS:
        cs_BuildOffsets::clearMode = 1u;
        dispatch(grid_groups, par, [](uint g) {
            cs_BuildOffsets::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_BuildOffsets::main();
        });
        cs_BuildOffsets::clearMode = 0u;
        dispatch(groups, par, [](uint g) {
            cs_BuildOffsets::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_BuildOffsets::main();
        });
        return 0;
    case GLSL_LOD:
        dispatch(groups, par, [](uint g) {
            cs_ComputeLOD::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_ComputeLOD::main();
        });
        return 0;
    case GLSL_LAMBDAS:
        cs_ComputeLambdas::currentIter = iter;
        dispatch(groups, par, [](uint g) {
            cs_ComputeLambdas::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_ComputeLambdas::main();
        });
        return 0;
    case GLSL_DELTAP:
        cs_ComputeDeltaP::currentIter = iter;
        dispatch(groups, par, [](uint g) {
            cs_ComputeDeltaP::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_ComputeDeltaP::main();
        });
        return 0;
    case GLSL_APPLY:
        cs_ApplyDeltaP::currentIter = iter;
        dispatch(groups, par, [](uint g) {
            cs_ApplyDeltaP::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_ApplyDeltaP::main();
        });
        return 0;
    case GLSL_INTEGRATE: {
        std::vector<cs_Integrate::Particle> snap;
        if (c->pre_integrate) {
            snap.assign((cs_Integrate::Particle*)c->particles, (cs_Integrate::Particle*)c->particles + N);
            cs_Integrate::particles_prev = snap.data();
        } else {
            cs_Integrate::particles_prev = (cs_Integrate::Particle*)c->particles;
        }
        dispatch(groups, par, [](uint g) {
            cs_Integrate::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_Integrate::main();
        });
        cs_Integrate::particles_prev = (cs_Integrate::Particle*)c->particles;
        return 0;
    }
    case GLSL_VORTICITY:
        dispatch(groups, par, [](uint g) {
            cs_VorticityConfinement::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_VorticityConfinement::main();
        });
        return 0;
    case GLSL_CONTACT:
        *c->contact_count = 0;
        dispatch(groups, false, [](uint g) {
            cs_ContactFilter::gl_GlobalInvocationID = uvec3{g, 0, 0};
            cs_ContactFilter::main();
        });
        return 0;
    default:
        return -1;
    }
}

}  // namespace

extern "C" int glsl_ref_stage(glsl_ref_ctx* c, int stage, uint32_t iter)
{
    bind_all(c);
    return run_stage(c, stage, iter);
}

// PBFluids::step (src/fluid/PBFluids.cpp:323-517)
extern "C" int glsl_ref_step(glsl_ref_ctx* c)
{
    if (c->n == 0) return 0;
    bind_all(c);
    const uint32_t max_iter = c->ubo.enable_apbf ? c->ubo.max_lod : c->solver_iterations;
    for (uint32_t s = 0; s < c->substeps; ++s) {
        run_stage(c, GLSL_PREDICT, 0);
        run_stage(c, GLSL_SORT, 0);
        run_stage(c, GLSL_OFFSETS, 0);
        if (c->ubo.enable_apbf) run_stage(c, GLSL_LOD, 0);
        for (uint32_t it = 1; it <= max_iter; ++it) {
            run_stage(c, GLSL_LAMBDAS, it);
            run_stage(c, GLSL_DELTAP, it);
            run_stage(c, GLSL_APPLY, it);
        }
        run_stage(c, GLSL_INTEGRATE, 0);
    }
    if (c->enable_vorticity) run_stage(c, GLSL_VORTICITY, 0);
    return 0;
}
