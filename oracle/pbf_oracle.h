/*
 * pbf_oracle.h — FP64 CPU restatement of the reference PBF substep (and its
 * float32 build, see orc_real below).
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product path links or calls this
 * code: it is the checker used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py.
 *
 * Each function restates one reference compute shader or host routine of
 * enderenest/Realtime-FSI-Engine and cites it by path:line.  State is held in
 * particle (original id) order, exactly as the reference does: the hash grid
 * is a list of (key, id) pairs sorted stably by key, and neighbour loops go
 * through the id column (hashGrid[k].y).
 *
 * Parity pinning: the kernel functions and the hash/27-bucket neighbour
 * semantics are checked against the reference's own CPU code
 * (src/fluid/Kernels.cpp, src/fluid/NeighborSearch.cpp) and the per-dispatch
 * shader math against the reference GLSL compiled as C++ (oracle/glsl), both
 * built under oracle/_ref and frozen into tests/golden by
 * tests/golden/make_golden.py.
 *
 * Semantics fixed by this oracle (the defined behaviour of the drop-in):
 *   - stale grid: buckets come from predict-time x*, lookups use current x_i;
 *   - 27 hashed buckets with multiplicity (colliding neighbour cells are
 *     visited twice, as the shader loop does);
 *   - CS_Integrate reads neighbour velocities from before the dispatch (the
 *     reference reads particles[j].vel while other invocations write it,
 *     CS_Integrate.glsl:171 vs :277 — a race; pre-integrate is the defined
 *     choice);
 *   - SDF sampling is exact trilinear with clamp-to-edge, texel centre i at
 *     origin + i*cell (GL_LINEAR's 8-bit weights are not reproduced).
 */
#ifndef PBF_ORACLE_H
#define PBF_ORACLE_H

#include <stdint.h>
#include "../include/pbf_b200.h"

/* The oracle's arithmetic type: double for the FP64 restatement
 * (liboracle.so).  Built with -DORC_REAL=float it is the same algorithm with
 * float32 storage and sequential sums (liboracle32.so): the reference for
 * what FP32 arithmetic itself achieves on a computation, against which the
 * GPU's FP32 results are judged where FP32 rounding is amplified (the
 * 16-substep adjoint). */
#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL orc_real;

#ifdef __cplusplus
extern "C" {
#endif

/* FP64 copy of the FluidConfigUBO block plus the per-step settings that the
 * reference passes as shader uniforms. */
typedef struct orc_params {
    orc_real bmin[3], bmax[3], g[3];
    orc_real dt; /* substep dt: FluidConfig::dt / substepIterations */
    orc_real h, h2, rho0, eps, wq;
    orc_real k_corr, n_corr, viscosity, damping, cohesion;
    orc_real i_radius, i_strength;
    orc_real w0_self, poly6, spiky, inv_rho0;
    orc_real vort_eps, lod_max_dist;
    uint32_t hash_size, mask;
    uint32_t scorr, visc_on, vort_on, apbf, min_lod, max_lod;
    uint32_t iterations, substeps;
    uint32_t interacting;
    orc_real i_pos[3];
    orc_real camera[3];
} orc_params;

/* A sampled signed-distance grid (SDFBoundary data, SDFBoundary.h:128-131). */
typedef struct orc_sdf {
    int enabled;
    int dims[3];
    orc_real origin[3];
    orc_real cell;
    const float* dist; /* index(x,y,z) = x*dy*dz + y*dz + z */
    orc_real padding;
    int containment;
} orc_sdf;

/* PBFluids::setParams / setBounds (src/fluid/PBFluids.cpp:39-109,299-306) */
void orc_derive(const pbf_fluid_config* c, orc_real collision_padding, orc_params* p);

/* getGridHash (CS_PredictAndHash.glsl:77-83) */
uint32_t orc_hash(int32_t cx, int32_t cy, int32_t cz, uint32_t mask);
/* cell = ivec3(floor(x / h)) in FP32 as the shader computes it
 * (CS_PredictAndHash.glsl:125); x4 is float4-strided. */
void orc_keys_f32(const float* x4, uint32_t n, float h, uint32_t mask, uint32_t* keys);

/* Stable sort of (key, id), ids 0..n-1 in input order — the contract of the
 * LSD radix chain CS_RadixHistogram/PrefixSum/Scatter (PBFluids.cpp:354-405). */
void orc_stable_sort(const uint32_t* keys, uint32_t n, uint32_t hash_size, uint32_t* sorted_keys,
                     uint32_t* sorted_ids);
/* CS_BuildOffsets.glsl:55-78 (clear to -1, then start/end exclusive). */
void orc_build_table(const uint32_t* sorted_keys, uint32_t n, uint32_t hash_size, int32_t* table);

/* Trilinear clamp-to-edge SDF sample and central-difference gradient
 * (CS_Integrate.glsl:86-99, CS_ApplyDeltaP.glsl:53-65). */
orc_real orc_sdf_query(const orc_sdf* s, const orc_real p[3]);
void orc_sdf_gradient(const orc_sdf* s, const orc_real p[3], orc_real g[3]);

/* --- per-dispatch passes; arrays are particle-order orc_real[n][3] --------- */
/* CS_PredictAndHash.glsl:88-130.  vel is updated in place; keys from FP64 x*. */
void orc_predict(const orc_params* p, uint32_t n, const orc_real* pos, orc_real* vel, orc_real* xstar,
                 uint32_t* keys);
/* CS_ComputeLOD.glsl:66-79 */
void orc_lod(const orc_params* p, uint32_t n, const orc_real* xstar, uint32_t* lod);
/* CS_ComputeLambdas.glsl:108-162.  lod may be NULL. */
void orc_lambda(const orc_params* p, uint32_t n, const orc_real* xstar, const uint32_t* sorted_ids,
                const int32_t* table, const uint32_t* lod, uint32_t iter, orc_real* lambda,
                orc_real* rho);
/* CS_ComputeDeltaP.glsl:120-166 then CS_ApplyDeltaP.glsl:80-124 (two
 * dispatches: every Δp is computed from the same x* before any is applied). */
void orc_deltap_apply(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* xstar,
                      const orc_real* lambda, const uint32_t* sorted_ids, const int32_t* table,
                      const uint32_t* lod, uint32_t iter, orc_real* dp_out);
/* CS_Integrate.glsl:135-280 with pre-dispatch neighbour velocities. */
void orc_integrate(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* pos, orc_real* vel,
                   const orc_real* xstar, const uint32_t* sorted_ids, const int32_t* table,
                   orc_real* omega);
/* CS_VorticityConfinement.glsl:133-167 (pass 1, PBFluids.cpp:499-505). */
void orc_vorticity(const orc_params* p, uint32_t n, const orc_real* pos, orc_real* vel,
                   const orc_real* omega, const uint32_t* sorted_ids, const int32_t* table);

/* PBFluids::step (src/fluid/PBFluids.cpp:323-517) in FP64.  Optional outputs
 * (may be NULL): omega/rho of the last substep, sorted keys/ids and table of
 * the last substep (table needs 2*hash_size int32). */
void orc_step(const orc_params* p, const orc_sdf* s, uint32_t n, orc_real* pos, orc_real* vel,
              orc_real* omega, orc_real* rho, uint32_t* sorted_keys, uint32_t* sorted_ids,
              int32_t* table);

/* Reverse-mode derivative of orc_step (pbf_adjoint.c): from the adjoints of
 * the final positions/velocities (gpos/gvel, may be NULL = zero) to those of
 * the initial state (gpos0/gvel0) and of the SDF translation (gt, the origin
 * offset already applied to s).  pos_out/vel_out (may be NULL) receive the
 * forward result.  APBF and the interaction force must be off. */
void orc_adjoint_step(const orc_params* p, const orc_sdf* s, uint32_t n, const orc_real* pos0, const orc_real* vel0,
                      const orc_real* gpos, const orc_real* gvel, orc_real* gpos0, orc_real* gvel0, orc_real* gt,
                      orc_real* pos_out, orc_real* vel_out);

/* CS_ContactFilter.glsl:68-83, deterministic (particle order).  Returns the
 * count; out_idx receives the particle ids. */
uint32_t orc_contact_filter(const orc_sdf* s, uint32_t n, const orc_real* pos, orc_real band,
                            uint32_t* out_idx);

/* poly6 value and spiky gradient at offset r (CS_ComputeLambdas.glsl:74-92). */
void orc_kernels(const orc_params* p, const orc_real r[3], orc_real* w, orc_real g[3]);
/* In-range visited candidates per particle (NeighborSearch.cpp:97-126 semantics). */
void orc_neighbor_lists(const orc_params* p, uint32_t n, const orc_real* x, const uint32_t* ids,
                        const int32_t* table, int32_t* counts, int32_t* lists, int32_t cap);

/* ---- triangle-mesh SDF (src/fluid/SDFBoundary.cpp) ----------------------- */
typedef struct orc_mesh orc_mesh;
/* SDFBoundary::buildFromMesh (SDFBoundary.cpp:278-398) minus the grid fill. */
orc_mesh* orc_mesh_build(const orc_real* verts, int32_t nv, const int32_t* faces, int32_t nf,
                         orc_real cell);
void orc_mesh_free(orc_mesh* m);
/* SDFBoundary::updateGeometryAndRefit (SDFBoundary.cpp:438-453). */
void orc_mesh_refit(orc_mesh* m, const orc_real* verts);
void orc_mesh_grid_info(const orc_mesh* m, int32_t dims[3], orc_real origin[3], orc_real* cell);
/* SDFBoundary::recomputeDistances (SDFBoundary.cpp:421-436) into out (size
 * dx*dy*dz, index() order). */
void orc_mesh_grid(const orc_mesh* m, float* out);
/* SDFBoundary::signedDistanceAt (SDFBoundary.cpp:400-419). */
orc_real orc_mesh_signed_distance(const orc_mesh* m, const orc_real p[3]);
/* TriangleBVH::closestPoint (SDFBoundary.cpp:151-155,225-257): face index,
 * closest point, squared distance. */
int32_t orc_mesh_closest(const orc_mesh* m, const orc_real p[3], orc_real point[3], orc_real* dist2);
/* computeContactForces (src/main.cpp:604-710) in FP64 with a fixed
 * (candidate-order) summation.  cand: count ContactCandidate records. */
int32_t orc_contact_forces(const orc_mesh* m, const pbf_contact_candidate* cand, uint32_t count,
                           orc_real band, int use_vel_magnitude, orc_real* forces3);

#ifdef __cplusplus
}
#endif
#endif
