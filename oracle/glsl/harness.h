/*
 * harness.h — C interface of the reference-shader CPU harness
 * (oracle/_ref/libpbfref_glsl.so, built by oracle/Makefile from the
 * reference's resources/shaders/compute/*.glsl via oracle/glsl/translate.py).
 *
 * TEST INFRASTRUCTURE ONLY.  Buffers are in the reference's GPU layouts:
 * Particle {vec4 pos, predPos, vel} (48 B), SolverData {vec4 predPos_lambda,
 * deltaP_rho} (32 B), hashGrid uvec2 (hash, id), offsets ivec2 per hash,
 * ContactCandidate {vec4 pos, vel}.
 */
#ifndef PBF_GLSL_HARNESS_H
#define PBF_GLSL_HARNESS_H
#include <stdint.h>
#include "../../include/pbf_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct glsl_ref_ctx {
    pbf_derived_params ubo; /* FluidConfigUBO contents (std140 compatible) */
    uint32_t n;
    void* particles;         /* n * 48 B                  */
    void* solver;            /* n * 32 B                  */
    uint32_t* hash_grid;     /* 2n                        */
    uint32_t* hash_grid_alt; /* 2n                        */
    uint32_t* histogram;     /* 256 * ceil(n/256)         */
    int32_t* offsets;        /* 2 * hash_size             */
    uint32_t* lod;           /* n                         */
    uint32_t* contact_count; /* 1                         */
    void* contacts;          /* n * 32 B                  */
    uint32_t is_interacting;
    float interaction_pos[3];
    float camera_pos[3];
    uint32_t enable_vorticity;
    float vorticity_epsilon;
    uint32_t enable_sdf;
    uint32_t sdf_mode;
    const float* sdf_dist; /* CPU order x*dy*dz + y*dz + z */
    int32_t sdf_dims[3];
    float sdf_origin[3];
    float sdf_cell;
    float sdf_padding;
    float contact_band;
    uint32_t substeps;
    uint32_t solver_iterations;
    int32_t sort_mode;     /* 0: std::stable_sort by key, 1: emulate the radix shaders */
    int32_t parallel;      /* OpenMP over invocations of barrier-free dispatches        */
    int32_t pre_integrate; /* CS_Integrate reads the pre-dispatch velocity snapshot      */
} glsl_ref_ctx;

enum glsl_ref_stage {
    GLSL_PREDICT = 1,
    GLSL_SORT = 2,
    GLSL_OFFSETS = 3,
    GLSL_LOD = 4,
    GLSL_LAMBDAS = 5,
    GLSL_DELTAP = 6,
    GLSL_APPLY = 7,
    GLSL_INTEGRATE = 8,
    GLSL_VORTICITY = 9,
    GLSL_CONTACT = 10
};

/* One dispatch (or the 4-pass radix chain for GLSL_SORT) as PBFluids::step
 * issues it; `iter` is the 1-based solver iteration uniform. */
int glsl_ref_stage(glsl_ref_ctx* c, int stage, uint32_t iter);
/* PBFluids::step (src/fluid/PBFluids.cpp:323-517). */
int glsl_ref_step(glsl_ref_ctx* c);

#ifdef __cplusplus
}
#endif
#endif
