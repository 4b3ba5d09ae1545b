// pbf_batch.h — the multi-scene engine behind the pbf_batch_* C ABI.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/pbf_b200.h"
#include "pbf_kernels.h"

namespace pbf {

// Per-scene constants read by the multi-scene passes (device array, one
// entry per scene).
struct SceneDev {
    uint32_t table_off;  // first bucket of the scene in the shared cell table
    uint32_t mask;       // H_k - 1
    float bmin[3], bmax[3];  // walls after collision padding (PBFluids::setBounds)
    int cell_lo[3];      // lowest cell of the walls: origin of the Morton code
    int pad_;
    SdfDev sdf;
    // dense window (neighbour mode 8): cell of window slot (0, 0, 0), extent,
    // first global slot
    int win_g0[3];
    uint32_t win_n[3];
    uint32_t slot0;
};

#ifdef __CUDACC__
// The SDF of scene S as the passes sample it.
__device__ __forceinline__ SdfDev load_sdf(const SceneDev* S)
{
    SdfDev d;
    d.enabled = __ldg(&S->sdf.enabled);
    d.dist = S->sdf.dist;
    d.slab_min = S->sdf.slab_min;
    d.dx = __ldg(&S->sdf.dx);
    d.dy = __ldg(&S->sdf.dy);
    d.dz = __ldg(&S->sdf.dz);
    d.ox = __ldg(&S->sdf.ox);
    d.oy = __ldg(&S->sdf.oy);
    d.oz = __ldg(&S->sdf.oz);
    d.cell = __ldg(&S->sdf.cell);
    d.inv_cell = __ldg(&S->sdf.inv_cell);
    d.padding = __ldg(&S->sdf.padding);
    d.containment = __ldg(&S->sdf.containment);
    return d;
}
#endif

struct BatchLaunch {
    int block = 128;         // threads per block of the neighbour passes
    int blocks_per_sm = 0;   // persistent grid (0: one thread per particle)
    int sms = 148;
};

void launch_b_predict(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const float4* pos,
                      const float4* vel, uint32_t* keys, int sms, cudaStream_t st);
void launch_b_reorder(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* ids,
                      const float4* pos, const float4* vel, float4* sx, float4* sv, float4* sx0, uint32_t* lod,
                      uint32_t* mcode, uint32_t mbits, int sms, cudaStream_t st);
void launch_b_lambda(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                     const float4* xin, float4* xout, float* rho, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, cudaStream_t st);
void launch_b_deltap(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                     const float4* xin, float4* xout, const int2* table, const uint32_t* lod, uint32_t iter,
                     const uint32_t* order, cudaStream_t st);
void launch_b_integrate(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                        const float4* xs, const float4* sv, float4* sx0, float4* somega, const uint32_t* ids,
                        float4* pos, float4* vel, const int2* table, const uint32_t* order, cudaStream_t st);
void launch_b_vorticity(const DevParams& P, const BatchLaunch& L, const SceneDev* scenes, const uint16_t* scene_of,
                        const float4* spos, const float4* somega, const uint32_t* ids, float4* vel, const int2* table,
                        const uint32_t* order, cudaStream_t st);
int batch_max_blocks_per_sm(int block);

// ---- k_adjoint.cu ---------------------------------------------------------------------------
void launch_ad_lambda_rec(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                          const int2* table, const float4* xin, float4* xl, float4* auxl, float* rhol, cudaStream_t st);
void launch_ad_deltap_rec(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                          const int2* table, const float4* xl, float4* xout, float4* auxd, cudaStream_t st);
void launch_ad_vorticity(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                         const int2* table, const float4* spos, const float4* somega, const uint32_t* ids,
                         const float4* velb, float4* posb_s, float4* omb, cudaStream_t st);
void launch_ad_integrate(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                         const int2* table, const float4* xs, const float4* sv, const float4* cp_pos,
                         const uint32_t* ids, const float4* posb, const float4* velb, const float4* posb_s,
                         const float4* omb, const float4* somega, float4* gx, float4* gv, float4* x0b, float* tgrad,
                         cudaStream_t st);
void launch_ad_deltap(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                      const int2* table, const float4* xl, const float4* auxd, const float4* gin, float4* gout,
                      float* tgrad, cudaStream_t st);
void launch_ad_lambda(const DevParams& P, const SceneDev* scenes, const uint16_t* scene_of, const uint32_t* order,
                      const int2* table, const float4* xl, const float4* auxl, const float* rhol, float4* gout,
                      cudaStream_t st);
void launch_ad_predict(uint32_t n, float dt, const uint32_t* ids, const float4* gx, const float4* gv,
                       const float4* x0b, float4* posb, float4* velb, int sms, cudaStream_t st);

}  // namespace pbf

struct pbf_batch {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;

    pbf_fluid_config cfg{};        // shared solver constants
    pbf_derived_params derived{};  // of cfg (walls per scene)
    float collision_padding = 0.0f;

    struct Scene {
        pbf_scene_desc desc{};
        uint32_t offset = 0, table_off = 0;
        float* grid = nullptr;
        float* slab_min = nullptr;
        int dims[3] = {0, 0, 0};
        float origin[3] = {0, 0, 0};
        float cell = 0.0f;
        bool sdf_on = false;
        float sdf_padding = 0.0f;
        bool containment = false;
        float sdf_offset[3] = {0, 0, 0};  // translation of the SDF (differentiable pose)
    };
    std::vector<Scene> scenes;
    uint32_t n = 0;            // total particles
    uint32_t table_size = 0;   // sum of H_k
    uint32_t key_bits = 1;     // bits of the offset hash keys
    uint32_t mbits = 8;        // Morton bits per axis
    uint32_t order_bits = 24;  // bits of the scene-prefixed Morton keys

    // particle order
    float4 *pos = nullptr, *vel = nullptr, *pred = nullptr, *aos = nullptr;
    uint16_t* scene_of = nullptr;
    pbf::SceneDev* scenes_dev = nullptr;
    uint32_t* keys = nullptr;
    uint32_t *ka = nullptr, *ia = nullptr, *kb = nullptr, *ib = nullptr;
    uint32_t *skeys = nullptr, *ids = nullptr;
    uint32_t *hist = nullptr, *totals = nullptr;
    int2* table = nullptr;
    uint32_t *mcode = nullptr, *mka = nullptr, *mia = nullptr, *mkb = nullptr, *mib = nullptr;
    uint32_t* order = nullptr;
    // sorted order
    float4 *sx[2] = {nullptr, nullptr}, *sv = nullptr, *sx0 = nullptr, *somega = nullptr;
    float4* dpb = nullptr;  // lambda-independent part of each delta-p sum (DevParams::dpb)
    float* rho = nullptr;
    uint32_t* lod = nullptr;
    // autotuner state snapshot
    float4 *save_pos = nullptr, *save_vel = nullptr;

    // options (PBF_BOPT_*)
    pbf::BatchLaunch launch{};
    int morton = 1;
    bool use_graph = true;
    int neighbour_mode = -1;  // -1 automatic, 4 hashed buckets, 8 dense windows
    int tuned_mode = 0;       // the autotuner's pick under -1 (0: none yet)

    // neighbour mode 8 (k_dense.cu): a dense cell window per scene, scene k's
    // window at global slots [SceneDev::slot0, + its cells); labels sorted by
    // (global slot of the predict-time cell, hash-sorted index), scene-contiguous
    std::vector<int> win;         // per scene: g0[3], n[3], slot0 (7 ints), as uploaded
    uint64_t dense_total = 0;     // slots of all windows
    bool dense_ready = false;     // the clean/dcol tables below match `win` and the hash masks
    float4 *lx[2] = {nullptr, nullptr}, *lxb = nullptr, *lv = nullptr, *lx0 = nullptr, *lom = nullptr;
    float* lrho = nullptr;
    uint32_t *lid = nullptr, *lkey = nullptr, *inv = nullptr;
    int2 *dtable = nullptr, *druns = nullptr;
    uint16_t* dclean = nullptr;
    uint32_t* ddirty = nullptr;
    uint8_t *ddcol = nullptr, *dhcnt = nullptr, *dvmark = nullptr;
    uint16_t* dslot_scene = nullptr;
    uint32_t *dflag = nullptr, *dslot = nullptr, *dord = nullptr, *dcnt = nullptr, *dbsum = nullptr;
    uint32_t* dhm = nullptr;

    uint64_t launches = 0;
    bool capturing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t graph_launches = 0;

    // adjoint (pbf_adjoint.cu): per-substep checkpoints of the recorded step,
    // per-iteration recomputation buffers, adjoint accumulators
    uint32_t ad_subs = 0, ad_iters = 0;
    bool recorded = false;
    float4 *cp_pos = nullptr, *cp_vel = nullptr;       // substeps x n, particle order
    float4 *xl = nullptr, *auxl = nullptr, *auxd = nullptr;  // iterations x n, sorted
    float* rhol = nullptr;                              // iterations x n
    float4 *gxa = nullptr, *gxb = nullptr, *gv = nullptr, *x0b = nullptr;  // sorted
    float4 *pb = nullptr, *vb = nullptr;                // particle order
    float4 *pbs = nullptr, *omb = nullptr;              // sorted (vorticity reverse)
    float4 *tpos = nullptr, *tvel = nullptr;            // particle-order scratch of the recompute
    float* tgrad = nullptr;                             // 4 per scene
    cudaGraph_t rec_graph = nullptr, bwd_graph = nullptr;
    cudaGraphExec_t rec_exec = nullptr, bwd_exec = nullptr;
    uint64_t rec_launches = 0, bwd_launches = 0;

    ~pbf_batch();
    pbf::DevParams dev_params() const;
    bool dense_fits() const { return dense_total > 0 && dense_total <= (1ull << 26) && !derived.enable_apbf; }
    int effective_mode() const;
    int dense_setup();
    void dense_free();
    pbf::DenseArgs dense_args() const;
    int dense_step_body();
    int upload_scenes();
    void invalidate_graph();
    int step_body();
    int step();
    int substep_body(const float4* src_pos, const float4* src_vel, float4* dst_pos, float4* dst_vel);
    int ad_alloc();
    void ad_free();
    int record_body();
    int backward_body();
};
