/*
 * pbf_b200.h — C ABI of the B200 (sm_100a) position-based-fluids substep engine.
 *
 * This is the drop-in boundary for the fluid-solver hot path of
 * enderenest/Realtime-FSI-Engine.  The reference exposes that path only as the
 * C++ class `PBFluids` (include/fluid/PBFluids.h:88-163) plus the
 * `SDFBoundary` obstacle (include/fluid/SDFBoundary.h:38-167) and the
 * fluid-to-mesh contact reduction in src/main.cpp:604-710.  Every entry point
 * below names the reference member or function it replaces.  The C++ classes
 * in include/fluid/ (PBFluids.h, SDFBoundary.h) are thin wrappers over these functions.
 *
 * Conventions
 *   - Every function returns an int status: PBF_OK (0) or a negative PBF_ERR_*.
 *     pbf_last_error() returns a text description of the last failure on the
 *     calling thread.  No C++ exception crosses this boundary.
 *   - A handle owns one CUDA stream and all device buffers of one scene.  A
 *     handle is not thread-safe; distinct handles are independent.
 *   - Host pointers are plain host memory (pageable or pinned).  Sizes are in
 *     elements unless a name ends in _bytes.
 *   - pbf_step() is asynchronous on the handle's stream; every pbf_read_*()
 *     synchronizes the stream before it returns.
 */
#ifndef PBF_B200_H
#define PBF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PBF_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------- */
#define PBF_OK 0
#define PBF_ERR_INVALID -1   /* bad argument (null pointer, size, range)       */
#define PBF_ERR_CUDA -2      /* a CUDA runtime call failed                      */
#define PBF_ERR_STATE -3     /* call not valid in the current handle state      */
#define PBF_ERR_ALLOC -4     /* device or host allocation failed               */
#define PBF_ERR_NUMERIC -5   /* NaN/Inf detected in particle state             */
#define PBF_ERR_TIMEOUT -6   /* a bounded device-side wait gave up             */
#define PBF_ERR_NOT_BUILT -7 /* feature compiled out / library missing          */

/* ---- plain-C mirrors of the reference's POD types ------------------------ */

/* FluidConfig (include/core/config.h:9-63).  Field order, meaning and the
 * defaults filled in by pbf_default_config() follow the reference struct;
 * booleans are uint32_t (0/1) so the layout is fixed for every FFI. */
typedef struct pbf_fluid_config {
    float dt;                  /* macro time step                               */
    float gravity[3];
    float h;                   /* smoothing radius                              */
    float rho0;                /* rest density (unit particle mass implied)     */
    uint32_t solver_iterations;
    uint32_t substep_iterations;
    float eps;                 /* CFM relaxation epsilon                        */
    uint32_t particle_count;
    float spawn_min[3];
    float spawn_max[3];
    uint32_t spawn_random;
    float spacing;
    float initial_velocity[3];
    float bounds_min[3];
    float bounds_max[3];
    float bound_damping;
    uint32_t hash_size;        /* must be a power of two                        */
    uint32_t enable_scorr;
    float k_corr;
    float n_corr;
    float delta_q;
    float cohesion_strength;
    uint32_t enable_viscosity;
    float viscosity;
    float interaction_radius;
    float interaction_strength;
    uint32_t enable_vorticity;
    float vorticity_epsilon;
    uint32_t enable_apbf;
    uint32_t min_lod;
    uint32_t max_lod;
    float lod_max_dist;
} pbf_fluid_config;

/* Particle (include/fluid/Particle.h:8-12): three vec3 each padded to 16 B. */
typedef struct pbf_particle {
    float pos[3];
    float pad0;
    float pred_pos[3];
    float pad1;
    float vel[3];
    float pad2;
} pbf_particle;

/* ContactCandidate (include/fluid/PBFluids.h:67-70). */
typedef struct pbf_contact_candidate {
    float pos[4]; /* xyz world position, w unused */
    float vel[4]; /* xyz velocity, w unused       */
} pbf_contact_candidate;

/* Derived solver constants: the FluidConfigUBO block of
 * include/fluid/PBFluids.h:21-61 as PBFluids::setParams
 * (src/fluid/PBFluids.cpp:39-109) fills it. */
typedef struct pbf_derived_params {
    float bounds_min[4];
    float bounds_max[4];
    float gravity_dt[4]; /* xyz gravity, w substep dt */
    float h, rho0, eps, wq;
    float k_corr, n_corr, viscosity, bound_damping;
    uint32_t hash_size, particle_count, enable_scorr, enable_viscosity;
    float cohesion_strength, interaction_radius, interaction_strength, w0_self;
    uint32_t hash_mask;
    float poly6_coeff, spiky_coeff, inv_rho0;
    uint32_t min_lod, max_lod;
    float lod_max_dist;
    uint32_t enable_apbf;
} pbf_derived_params;

typedef struct pbf_handle pbf_handle;

/* ---- library ------------------------------------------------------------ */
int pbf_abi_version(void);
const char* pbf_last_error(void);
/* FluidConfig's in-class defaults (include/core/config.h:11-62). */
int pbf_default_config(pbf_fluid_config* out);
/* Host-side setParams derivation (src/fluid/PBFluids.cpp:39-109), exposed so
 * callers and tests see exactly the constants the kernels use.  `collision_padding`
 * is PBFluids::_collisionPadding (include/fluid/PBFluids.h:108-109). */
int pbf_derive_params(const pbf_fluid_config* cfg, float collision_padding,
                      pbf_derived_params* out);

/* ---- lifecycle (PBFluids::PBFluids / ~PBFluids, src/fluid/PBFluids.cpp:12-37) */
int pbf_create(const pbf_fluid_config* cfg, int device, pbf_handle** out);
int pbf_destroy(pbf_handle* h);

/* ---- parameters (PBFluids::setParams / setBounds / setCollisionPadding /
 *      setCameraPos / setInteraction, PBFluids.h:93-135, PBFluids.cpp:39-109,
 *      299-317) */
int pbf_set_params(pbf_handle* h, const pbf_fluid_config* cfg);
int pbf_get_params(pbf_handle* h, pbf_fluid_config* out);
int pbf_get_derived(pbf_handle* h, pbf_derived_params* out);
int pbf_set_bounds(pbf_handle* h, const float min_bound[3], const float max_bound[3],
                   float damping);
int pbf_set_collision_padding(pbf_handle* h, float padding);
int pbf_set_camera_pos(pbf_handle* h, const float pos[3]);
int pbf_set_interaction(pbf_handle* h, int active, const float pos[3]);

/* ---- particles (PBFluids::setParticles / readbackParticles,
 *      PBFluids.cpp:111-191).  n == 0 clears the scene (step() then no-ops,
 *      as PBFluids.cpp:325). */
int pbf_set_particles(pbf_handle* h, const pbf_particle* particles, uint32_t n);
/* Refresh the state of an unchanged particle count from host memory
 * (asynchronous on the handle's stream; pinned memory makes it a DMA).
 * No reference counterpart: setParticles also reallocates and re-derives. */
int pbf_upload_particles(pbf_handle* h, const pbf_particle* particles, uint32_t n);
int pbf_particle_count(pbf_handle* h, uint32_t* n);
int pbf_read_particles(pbf_handle* h, pbf_particle* out, uint32_t n);
/* Device-resident particle upload/download in the engine's own layout:
 * pos4 and vel4 are n float4 (xyz, w ignored) device pointers. */
int pbf_set_particles_device(pbf_handle* h, const void* pos4_dev, const void* vel4_dev,
                             uint32_t n);
int pbf_read_particles_device(pbf_handle* h, void* pos4_dev, void* vel4_dev, uint32_t n);

/* ---- stepping (PBFluids::step, PBFluids.cpp:323-517) ---------------------- */
int pbf_step(pbf_handle* h);
int pbf_sync(pbf_handle* h);
/* Raw cudaStream_t of the handle (for event timing / interop). */
int pbf_get_stream(pbf_handle* h, void** stream);

/* ---- SDF obstacle (PBFluids::setSDFBoundary / setSDFPadding /
 *      setSDFContainment, PBFluids.h:117-129; the sampled grid replaces
 *      SDFBoundary::uploadToGPU + Texture3D, SDFBoundary.cpp:580-598).
 *      `dist` is in the reference CPU order index(x,y,z) = x*dy*dz + y*dz + z
 *      (SDFBoundary.h:111-113); origin is the world position of voxel (0,0,0). */
int pbf_set_sdf_grid(pbf_handle* h, const float* dist, const int32_t dims[3],
                     const float origin[3], float cell_size);
int pbf_clear_sdf(pbf_handle* h);
/* Collide `h` with the SDF held by another handle `sdf` (same device) without
 * copying it: the non-owning pointer of PBFluids::setSDFBoundary
 * (PBFluids.h:117-120).  The caller keeps `sdf` alive while attached and
 * re-attaches after rebuilding it, as the reference does (main.cpp:852-854).
 * sdf == NULL detaches. */
int pbf_attach_sdf(pbf_handle* h, pbf_handle* sdf);
int pbf_set_sdf_mode(pbf_handle* h, float padding, int containment);
int pbf_read_sdf_grid(pbf_handle* h, float* out, size_t n);
/* Sample the active SDF at n world points (software trilinear, clamp to edge,
 * exactly as the step kernels query it).  out_grad may be NULL. */
int pbf_sample_sdf(pbf_handle* h, const float* pts3, uint32_t n, float* out_d,
                   float* out_grad3);

/* ---- triangle-mesh SDF (SDFBoundary::buildFromMesh / refitFromMesh /
 *      closestTriangle, SDFBoundary.cpp:278-465,600-610).  verts: nv*3 doubles,
 *      faces: nf*3 int32.  The grid is computed on the GPU from an LBVH and
 *      becomes the active SDF of the handle. */
int pbf_set_sdf_mesh(pbf_handle* h, const double* verts, int32_t nv, const int32_t* faces,
                     int32_t nf, double cell_size);
/* buildFromMesh again for moved vertices of the faces and cell size of the
 * last pbf_set_sdf_mesh (the reference's periodic full rebuild of a deforming
 * mesh, src/main.cpp:326): new grid origin and dimensions from the moved
 * bounding box, a new LBVH, face normals and the edge and angle-weighted
 * vertex pseudo-normals recomputed, the grid recomputed, all on the GPU (the
 * face-list adjacency from the first build is reused).  Same result as
 * pbf_set_sdf_mesh with these vertices. */
int pbf_rebuild_mesh(pbf_handle* h, const double* verts, int32_t nv);
/* Moved vertices, same topology: GPU LBVH refit + face-normal refresh + full
 * grid recompute (edge/vertex pseudo-normals keep their build-time values,
 * SDFBoundary.h:58-62). */
int pbf_update_mesh_vertices(pbf_handle* h, const double* verts, int32_t nv);
int pbf_sdf_grid_info(pbf_handle* h, int32_t dims[3], double origin[3], double* cell_size);
/* Closest point on the mesh for n query points (SDFBoundary::closestTriangle). */
int pbf_closest_triangle(pbf_handle* h, const float* pts3, uint32_t n, int32_t* out_face,
                         float* out_point3);

/* ---- contacts (PBFluids::filterContactCandidates / readbackContactCandidates,
 *      PBFluids.cpp:193-284; computeContactForces, src/main.cpp:604-710) ---- */
/* Near-surface compaction |sdf(x)| < band, in particle-index order (the
 * reference appends atomically in arbitrary order; this build is
 * deterministic).  band <= 0 or no SDF: no-op, as the reference. */
int pbf_filter_contacts(pbf_handle* h, float band);
int pbf_read_contacts(pbf_handle* h, pbf_contact_candidate* out, uint32_t capacity,
                      uint32_t* count);
/* Per-vertex fluid push forces from the current candidate list against the
 * current mesh: out3 receives nv*3 floats; out_contacts the number of
 * contributing candidates.  use_vel_magnitude mirrors g_useVelMagnitude. */
int pbf_vertex_forces(pbf_handle* h, float band, int use_vel_magnitude, float* out3,
                      int32_t nv, int32_t* out_contacts);

/* ---- stage-level access for parity tests -------------------------------- */
enum pbf_stage {
    PBF_STAGE_PREDICT = 1,   /* CS_PredictAndHash: keys (+ x*, v' recomputed later) */
    PBF_STAGE_SORT = 2,      /* CS_Radix*: stable sort of (key, id)                 */
    PBF_STAGE_TABLE = 3,     /* CS_BuildOffsets: clear + build the hash-cell table  */
    PBF_STAGE_REORDER = 4,   /* gather x*, v', x into sorted float4 SoA (+ LOD)     */
    PBF_STAGE_LAMBDA = 5,    /* CS_ComputeLambdas (iteration `iter`, 1-based)       */
    PBF_STAGE_DELTAP = 6,    /* CS_ComputeDeltaP + CS_ApplyDeltaP fused; reads the  */
                             /* per-particle sums PBF_STAGE_LAMBDA of the same      */
                             /* iteration wrote, so it runs after that stage        */
    PBF_STAGE_INTEGRATE = 7, /* CS_Integrate                                         */
    PBF_STAGE_VORTICITY = 8  /* CS_VorticityConfinement pass 1                       */
};
int pbf_run_stage(pbf_handle* h, int stage, uint32_t iter);

enum pbf_buffer {
    PBF_BUF_KEYS = 1,        /* uint32[N]  unsorted hash keys (particle order)      */
    PBF_BUF_SORTED_KEYS = 2, /* uint32[N]  sorted keys                              */
    PBF_BUF_SORTED_IDS = 3,  /* uint32[N]  particle id of each sorted slot          */
    PBF_BUF_TABLE = 4,       /* int32[2H]  (start, end) per hash, -1 if empty       */
    PBF_BUF_XSTAR = 5,       /* float4[N]  current (x*, lambda) in sorted order     */
    PBF_BUF_VPRED = 6,       /* float4[N]  post-predict velocity, sorted order      */
    PBF_BUF_RHO = 7,         /* float[N]   density of the last lambda pass, sorted  */
    PBF_BUF_OMEGA = 8,       /* float4[N]  curl omega of the last integrate, sorted */
    PBF_BUF_POS = 9,         /* float4[N]  committed positions, particle order      */
    PBF_BUF_VEL = 10,        /* float4[N]  committed velocities, particle order     */
    PBF_BUF_LOD = 11         /* uint32[N]  APBF level per sorted slot               */
};
int pbf_read_buffer(pbf_handle* h, int which, void* out, size_t bytes);
int pbf_buffer_device_ptr(pbf_handle* h, int which, void** dev_ptr, size_t* bytes);

/* ---- standalone primitives (host buffers in, host buffers out) ---------- */
/* Stable LSD radix sort of n keys < 2^key_bits with ids 0..n-1 — the contract
 * of the CS_RadixHistogram/PrefixSum/Scatter chain (PBFluids.cpp:354-405). */
int pbf_sort_keys(const uint32_t* keys, uint32_t n, uint32_t key_bits,
                  uint32_t* sorted_keys, uint32_t* sorted_ids);
/* CS_BuildOffsets (clear + build) over sorted keys into table[2*hash_size]. */
int pbf_build_table(const uint32_t* sorted_keys, uint32_t n, uint32_t hash_size,
                    int32_t* table);

/* Allocation-free variant of the stable (key, id) radix sort, for callers that
 * cannot call cudaMalloc (device memory owned by another framework's pool,
 * plugins handed only device buffers, real-time loops that must not enter the
 * allocator).  No counterpart in the reference.  keys_dev, sorted_keys_dev and
 * sorted_ids_dev are caller-owned device arrays of n uint32, no two of which
 * may overlap (PBF_ERR_INVALID otherwise); the work is queued on `stream` (a
 * cudaStream_t of the current device, NULL for the default stream; a stream of
 * another device gives PBF_ERR_INVALID) and the call returns without
 * synchronizing.  Scratch
 * comes from one fixed device array of the library (about 8.3 MB, kept by
 * every GPU that loads the library until exit), so n is limited to
 * PBF_NOALLOC_MAX_KEYS, and calls whose GPU work overlaps (other streams or
 * host threads) race on that array.  The first call on a device looks up the
 * array's device address; make it before capturing that device's streams into
 * a CUDA graph.  Keys wider than key_bits are ordered by their low key_bits. */
#define PBF_NOALLOC_MAX_KEYS (1u << 20)
int pbf_sort_keys_noalloc(const uint32_t* keys_dev, uint32_t n, uint32_t key_bits,
                          uint32_t* sorted_keys_dev, uint32_t* sorted_ids_dev, void* stream);

/* ---- timing ------------------------------------------------------------- */
/* When on, every pass of pbf_step records CUDA events on the handle's stream
 * and accumulates per-pass device time (read with pbf_read_pass_times).
 * Pass slots follow enum pbf_stage (index = stage); slot 0 = whole steps. */
#define PBF_NUM_PASS_SLOTS 12
int pbf_set_profiling(pbf_handle* h, int on);
int pbf_read_pass_times(pbf_handle* h, double* ms_out, uint64_t* launches_out);
int pbf_reset_pass_times(pbf_handle* h);
/* Number of kernels this library launched on the handle since creation. */
int pbf_kernel_launches(pbf_handle* h, uint64_t* out);
/* CUDA-graph replay of one full step (captured lazily, invalidated by any
 * parameter, particle or SDF change). */
int pbf_set_use_graph(pbf_handle* h, int on);
/* Execution options (results do not depend on them; no reference counterpart):
 *   PBF_OPT_SPATIAL_ORDER  the neighbour passes' walk.
 *                          4: particles taken in the Morton order of their
 *                          cells, one thread each, each of the 27 hashed
 *                          buckets tested in chunks of 8 before the pair body
 *                          runs on the hits.
 *                          8: data relabelled by the slot of each particle's
 *                          cell in a dense window of the box (z, y, x), so
 *                          the three x-adjacent cells of a row are one label
 *                          range: 9 runs replace the 27 buckets wherever the
 *                          cell's neighbourhood has no hash collision and no
 *                          particle within reach has moved 0.9 h since the
 *                          predict near a colliding cell; the hashed buckets
 *                          elsewhere.  Same pairs, same order as the buckets.
 *                          -1 (default): mode 8 from 2^19 particles, mode 4
 *                          below (where mode 8's relabelling launches cost
 *                          more than its walk saves); APBF and windows over
 *                          2^26 cells run mode 4.  Modes 4 and 8 give
 *                          bit-identical results (same pairs, order and pair
 *                          arithmetic).  Other values: PBF_ERR_INVALID. */
#define PBF_OPT_SPATIAL_ORDER 1
int pbf_set_option(pbf_handle* h, int option, int value);

/* Mode 8 statistics: particle passes that walked some rows of their
 * neighbourhood through the hashed buckets (since the window was set up),
 * particles beyond the 0.9 h drift bound that marked the cells within their
 * reach in the last substep (a same-bucket cell was near; counted per pass),
 * and window cells whose neighbourhood has a hash collision.  Zeros in
 * mode 4. */
int pbf_list_stats(pbf_handle* h, uint32_t* full_walks, uint32_t* bucket_walks, uint32_t* marked_buckets);

/* ---- health ------------------------------------------------------------- */
/* Scan committed state for NaN/Inf; *bad receives the count (0 = healthy). */
int pbf_check_finite(pbf_handle* h, uint32_t* bad);

/* ---- batched scenes ---------------------------------------------------------
 * No reference counterpart: the reference steps one scene per PBFluids
 * object (src/fluid/PBFluids.cpp:323-517).  A batch advances many independent
 * scenes of uneven particle counts that share the solver constants of one
 * pbf_fluid_config (h, dt, substeps, iterations, s_corr, XSPH, vorticity),
 * each with its own walls, hash size and SDF obstacle, by one launch per
 * pass over all scenes; the step is replayed from a CUDA graph.  Every scene
 * evolves exactly as a pbf_handle with the same configuration would (same
 * neighbour visitation, same per-pair arithmetic).  Not thread-safe per
 * batch; distinct batches are independent. */
typedef struct pbf_batch pbf_batch;

typedef struct pbf_scene_desc {
    uint32_t num_particles;
    uint32_t hash_size;      /* power of two; 0 = the shared config's hash_size */
    float bounds_min[3];     /* container walls, as FluidConfig::boundsMin/Max */
    float bounds_max[3];
} pbf_scene_desc;

#define PBF_BATCH_ALL 0xFFFFFFFFu /* scene index meaning "all scenes, concatenated" */

int pbf_batch_create(const pbf_fluid_config* cfg, const pbf_scene_desc* scenes, uint32_t num_scenes, int device,
                     pbf_batch** out);
int pbf_batch_destroy(pbf_batch* b);
/* Scene count and total particle count. */
int pbf_batch_info(const pbf_batch* b, uint32_t* num_scenes, uint32_t* total_particles);
/* First particle index of `scene` in the concatenated arrays and its count. */
int pbf_batch_scene_range(const pbf_batch* b, uint32_t scene, uint32_t* offset, uint32_t* count);
/* Wall padding of every scene (PBFluids::setCollisionPadding). */
int pbf_batch_set_collision_padding(pbf_batch* b, float padding);
/* Particles of one scene (n = its count) or, with PBF_BATCH_ALL, of all
 * scenes concatenated (n = total).  Velocities of the vorticity state are
 * reset as pbf_set_particles does. */
int pbf_batch_set_particles(pbf_batch* b, uint32_t scene, const pbf_particle* particles, uint32_t n);
int pbf_batch_read_particles(pbf_batch* b, uint32_t scene, pbf_particle* out, uint32_t n);
/* SDF obstacle of one scene: a distance grid in the layout of
 * pbf_set_sdf_grid; pbf_batch_set_sdf_mode sets its padding/containment. */
int pbf_batch_set_sdf_grid(pbf_batch* b, uint32_t scene, const float* dist, const int32_t dims[3],
                           const float origin[3], float cell);
int pbf_batch_set_sdf_mode(pbf_batch* b, uint32_t scene, float padding, uint32_t containment);
int pbf_batch_clear_sdf(pbf_batch* b, uint32_t scene);
/* One step() of every scene (substeps x iterations + vorticity), async. */
int pbf_batch_step(pbf_batch* b);
int pbf_batch_sync(pbf_batch* b);
int pbf_batch_get_stream(pbf_batch* b, void** stream);
/* Device arrays of the concatenated particles: float4 (x, pad0) and float4
 * (v, pad2) in particle order; valid until pbf_batch_destroy. */
int pbf_batch_device_ptrs(pbf_batch* b, void** pos4, void** vel4);
int pbf_batch_kernel_launches(const pbf_batch* b, uint64_t* count);

/* Options.  None changes results, only speed.
 *   PBF_BOPT_BLOCK          threads per block of the neighbour passes: 64, 128 (default), 256
 *   PBF_BOPT_ORDER          1 (default): threads take particles in the scene-prefixed
 *                           Morton order of their cells; 0: sorted (hash) order
 *   PBF_BOPT_BLOCKS_PER_SM  persistent grid of SMs x value blocks looping over the
 *                           particles; 0 (default): one thread per particle
 *   PBF_BOPT_USE_GRAPH      1 (default): replay the step from a CUDA graph
 *   PBF_BOPT_NEIGHBOUR_MODE -1 (default): automatic (the autotuner's pick once it has run,
 *                           before that 8 from 2^19 particles when the windows fit, else 4);
 *                           4: every scene walks its 27 hashed buckets (block, order and
 *                           persistence apply); 8: a dense cell window per scene (the walls'
 *                           box plus 6 cells each side, at most 2^26 cells in all, APBF off),
 *                           the passes of PBF_OPT_SPATIAL_ORDER mode 8 over all scenes at once.
 *                           Both give every scene the bits of its own pbf_handle. */
#define PBF_BOPT_BLOCK 1
#define PBF_BOPT_ORDER 2
#define PBF_BOPT_BLOCKS_PER_SM 3
#define PBF_BOPT_USE_GRAPH 4
#define PBF_BOPT_NEIGHBOUR_MODE 5
int pbf_batch_set_option(pbf_batch* b, int option, int value);
int pbf_batch_get_option(const pbf_batch* b, int option, int* value);

typedef struct pbf_batch_tuning {
    int32_t block;
    int32_t order;
    int32_t blocks_per_sm;
    float ms_per_step;
    int32_t neighbour_mode;  /* 4 or 8 (block, order and persistence apply to 4 only) */
} pbf_batch_tuning;
/* Times every candidate for `trial_steps` steps after one warm-up step, keeps
 * the fastest and restores the particle state that the trials advanced.  The
 * candidates: block x order x persistence in neighbour mode 4, and mode 8 when
 * the windows fit, as PBF_BOPT_NEIGHBOUR_MODE allows (-1: both; the pick then
 * decides the automatic mode).  `results` (may be null) receives up to
 * `max_results` timed candidates, `*num_results` their count; `*best` the pick. */
int pbf_batch_autotune(pbf_batch* b, uint32_t trial_steps, pbf_batch_tuning* best, pbf_batch_tuning* results,
                       uint32_t max_results, uint32_t* num_results);

/* ---- host deformation (the consumer of pbf_vertex_forces) -------------------
 * Cotangent-Laplacian surface deformation of a triangle mesh driven by
 * per-vertex handle targets: LaplacianDeformation (include/deformation/
 * LaplacianDeformation.h:11-157, src/deformation/LaplacianDeformation.cpp) and
 * the application's per-frame handle logic deformStep (src/main.cpp:870-944),
 * restated without Eigen/CHOLMOD/OpenMesh.  Host code, FP64 positions. */
typedef struct pbf_deform pbf_deform;

/* SceneDeform (include/core/Scene.h:17-27) / main.cpp's g_* tuning. */
typedef struct pbf_deform_params {
    float stiffness;             /* force -> displacement gain                  */
    float max_displacement;      /* per-frame displacement clamp                */
    float max_total_disp;        /* clamp on |deformed - rest|                  */
    uint32_t restore_enabled;    /* elastic spring-back toward rest             */
    float restore_strength;      /* fraction of the offset removed per frame    */
    float control_threshold;     /* |force| to enter the handle set             */
    float control_threshold_low; /* |force| to leave it (hysteresis)            */
} pbf_deform_params;

int pbf_deform_default_params(pbf_deform_params* out);
/* verts3: nv x 3 rest positions; faces3: nf x 3 vertex indices. */
int pbf_deform_create(const double* verts3, int32_t nv, const int32_t* faces3, int32_t nf, pbf_deform** out);
int pbf_deform_destroy(pbf_deform* d);
/* setUseLocal / setLocalKRing / setUseIncremental (defaults 1, 3, 0). */
int pbf_deform_set_mode(pbf_deform* d, int32_t use_local, int32_t kring, int32_t use_incremental);
int pbf_deform_add_anchor(pbf_deform* d, int32_t vertex);
int pbf_deform_set_control_points(pbf_deform* d, const int32_t* indices, const double* targets3, int32_t n);
int pbf_deform_precompute(pbf_deform* d);
int pbf_deform_solve(pbf_deform* d);
int pbf_deform_vertices(pbf_deform* d, double* out3, int32_t nv);
int pbf_deform_set_vertices(pbf_deform* d, const double* verts3, int32_t nv);
/* One frame: handle set from the forces (nv x 3), refactor when the set
 * changed, solve; *moved = 1 when the mesh was re-solved. */
int pbf_deform_step(pbf_deform* d, const float* forces3, int32_t nv, float dt, const pbf_deform_params* params,
                    int32_t* handle_count, int32_t* refactored, int32_t* moved);
int pbf_deform_patch_size(pbf_deform* d, int32_t* size);
/* Incremental path: max |x - x_dense| on the x axis (-1 if not ready). */
int pbf_deform_verify_incremental(pbf_deform* d, double* max_diff);

/* ---- scene presets and headless set-up (include/core/Scene.h,
 *      include/core/SceneSetup.h) --------------------------------------------
 * Host code, no GPU.  The presets are Scene.h:70-306's four scenes; the
 * set-up steps are the application's (src/main.cpp): loadOFF :364-415,
 * fitMeshToDomain :419-432, the fit centre of loadMeshBoundary :500-512,
 * applyMeshTransform :747-770, spawnParticles :160-188. */
typedef struct pbf_scene_preset {
    char name[48];
    pbf_fluid_config fluid;
    float cam_yaw, cam_pitch, cam_dist, point_size;
    char mesh_file[64];          /* asset file name, e.g. "cube1538.off"        */
    float mesh_fit_size;         /* largest extent after fitting                */
    float sdf_cell;              /* SDF voxel size                              */
    float sdf_padding;
    uint32_t sdf_container;      /* 1: fluid held inside the mesh               */
    float mesh_translate[3];     /* offset from the fitted pose                 */
    float mesh_rot_deg[3];       /* degrees about X, Y, Z (Rx * Ry * Rz)        */
    pbf_deform_params deform;    /* SceneDeform's first seven fields            */
    int32_t local_kring;         /* SceneDeform::localKRing                     */
    float contact_radius;        /* SceneDeform::contactRadius                  */
} pbf_scene_preset;

/* Number of presets (4). */
int pbf_scene_count(void);
int pbf_scene_get(int32_t index, pbf_scene_preset* out);
/* Reads an OFF mesh (comments and blank lines skipped, any *OFF header,
 * first three numbers of a vertex line, polygons fan-triangulated).  *nv and
 * *nf always receive the counts; verts3 (nv x 3) and faces3 (nf x 3) are
 * filled when their capacities (in vertices / triangles) suffice, so a
 * caller may ask for the counts first with null arrays. */
int pbf_off_load(const char* path, double* verts3, int32_t vcap, int32_t* faces3, int32_t fcap, int32_t* nv,
                 int32_t* nf);
/* Centre the bounding box on center and scale the largest extent to
 * target_size (in place). */
int pbf_mesh_fit(double* verts3, int32_t nv, const float center[3], double target_size);
/* The fit centre a scene uses: walls' middle in x and z, 40 % up in y. */
int pbf_mesh_fit_center(const pbf_fluid_config* cfg, float center_out[3]);
/* Rotate about the bounding-box centre (degrees, X then Y then Z) and
 * translate, in single precision (in place). */
int pbf_mesh_place(double* verts3, int32_t nv, const float translate[3], const float rot_deg[3]);
/* The reference's spawner for cfg (lattice, or seeded uniform with
 * spawn_random).  *count always receives the number of particles; `out` is
 * filled when capacity suffices. */
int pbf_spawn_particles(const pbf_fluid_config* cfg, pbf_particle* out, uint32_t capacity, uint32_t* count);

/* ---- differentiable step ----------------------------------------------------
 * No reference counterpart.  Reverse-mode derivative of one step of a batch
 * (all substeps x iterations, then vorticity) with respect to the initial
 * particle positions and velocities and each scene's SDF translation.  The
 * sort permutation and every discrete choice (neighbour sets, wall and SDF
 * contacts, clamps) are replayed from the recorded forward, not
 * differentiated.  Per-substep checkpoints of (x, v) are kept; the backward
 * recomputes each substep from its checkpoint.  APBF must be off.
 *
 * State arrays are n float4 (x, pad) / (v, pad) in the concatenated particle
 * order; pointers may be device or host memory (unified addressing). */
/* Translate scene `scene`'s SDF by t (the grid origin moves by t). */
int pbf_batch_set_sdf_offset(pbf_batch* b, uint32_t scene, const float t[3]);
int pbf_batch_set_state(pbf_batch* b, const void* pos4, const void* vel4);
int pbf_batch_get_state(pbf_batch* b, void* pos4, void* vel4);
/* One step exactly as pbf_batch_step, keeping what the backward needs. */
int pbf_batch_forward_record(pbf_batch* b);
/* Adjoint of the recorded step: gpos4/gvel4 (may be null = 0) are dL/d(final
 * x, v); out_gpos4/out_gvel4 (may be null) receive dL/d(initial x, v), out_gt
 * (may be null) 3 floats per scene, dL/d(SDF translation).  Synchronous. */
int pbf_batch_backward(pbf_batch* b, const void* gpos4, const void* gvel4, void* out_gpos4, void* out_gvel4,
                       float* out_gt);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* PBF_B200_H */
