// pbf_engine.h — the handle behind the C ABI (one scene, one stream).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/pbf_b200.h"
#include "pbf_kernels.h"

namespace pbf {
int set_error(int code, const char* fmt, ...);
}

struct pbf_handle {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;

    pbf_fluid_config cfg{};
    pbf_derived_params derived{};
    float collision_padding = 0.0f;
    bool interacting = false;
    float interaction_pos[3] = {0, 0, 0};
    float camera[3] = {0, 0, 0};

    uint32_t n = 0, cap_n = 0, cap_h = 0;

    // particle order
    float4* pos = nullptr;
    float4* vel = nullptr;
    float4* pred = nullptr;  // Particle::predPos + pad1, returned unchanged by readback
    float4* aos = nullptr;   // 3 float4 per particle: Particle staging for upload / readback
    uint32_t* keys = nullptr;
    // sort ping-pong; skeys/ids point into one pair after the sort
    uint32_t *ka = nullptr, *ia = nullptr, *kb = nullptr, *ib = nullptr;
    uint32_t* skeys = nullptr;
    uint32_t* ids = nullptr;
    uint32_t* hist = nullptr;
    uint32_t* totals = nullptr;
    int2* table = nullptr;
    // spatial processing order of the neighbour passes (Morton order of the
    // predict-time cells); `order` points into one of the m* ping-pong pairs.
    // PBF_OPT_SPATIAL_ORDER: 4 hashed buckets in Morton thread order with
    // per-bucket hit masks, 8 x-runs of the dense cell window; -1 (default): 8
    // from 2^19 particles, 4 below
    int pass_mode = -1;
    uint32_t *mcode = nullptr, *mka = nullptr, *mia = nullptr, *mkb = nullptr, *mib = nullptr;
    uint32_t* order = nullptr;
    // mode 8: the per-particle arrays relabelled by window slot
    float4 *lx[2] = {nullptr, nullptr}, *lxb = nullptr, *lv = nullptr, *lx0 = nullptr, *lom = nullptr;
    float* lrho = nullptr;
    uint32_t *lid = nullptr, *lkey = nullptr, *inv = nullptr;
    bool label_space = false;    // the current substep's state lives in the label arrays
    uint32_t cap_label_n = 0;
    // mode 8: runs of a dense cell window
    int2* dtable = nullptr;      // per window slot: label range
    int2* druns = nullptr;       // per window slot: label range of its x-run (slots s-1 .. s+1)
    uint16_t* dclean = nullptr;  // per window slot: rows whose buckets a hash collision near the cell affects
    uint8_t* ddcol = nullptr;    // per window slot: distance to the nearest other cell of its bucket
    uint32_t* ddirty = nullptr;  // per window slot: rows through which a moved particle is within reach (per substep)
    uint32_t* dflag = nullptr;   // [0] drift-bound crossings, [1] bucket walks, [2] unclean slots, [3] overflow labels
    // thread order of the passes after particles have moved (labels by current cell)
    uint32_t *dslot = nullptr, *dord = nullptr, *dcnt = nullptr, *dbsum = nullptr;
    uint32_t cap_ord_n = 0;
    int dord_iter = 0;           // solver iteration the order was computed for (0: none)
    bool dslot_fresh = false;    // dslot/dcnt hold the slots of the latest positions (recorded by a pass)
    // lambda hit masks replayed by the delta-p pass of the same iteration
    uint32_t* dhm = nullptr;
    uint8_t* dhcnt = nullptr;
    int dlist_iter = 0;          // solver iteration whose lambda recorded them (0: none)
    uint8_t* dvmark = nullptr;   // per window slot: integrate moved a particle its runs hold
    bool dvlist_ready = false;   // dhm/dhcnt hold the integrate pass's masks for the vorticity pass
    size_t cap_slots = 0;
    int dwin_g0[3] = {0, 0, 0};
    uint32_t dwin_n[3] = {0, 0, 0};
    uint32_t dwin_mask = 0;
    bool dwin_ready = false;
    uint32_t dwin_unclean = 0;
    // mode 8: the predict pass's window slot of each particle (particle order),
    // valid for the next relabelling when neither the particles (particles_gen),
    // the parameters nor the window changed in between
    uint32_t* dkey_id = nullptr;
    bool dkey_valid = false;
    uint64_t particles_gen = 0, dkey_gen = 0;
    pbf::DevParams dkey_P;
    int dkey_g0[3] = {0, 0, 0};
    uint32_t dkey_n[3] = {0, 0, 0};
    bool dense_window(int g0[3], uint32_t nd[3]) const;
    int ensure_dense();
    pbf::DenseArgs dense_args() const;
    int effective_mode() const;
    int ensure_label_capacity();
    int unpermute_for_read(int which);
    // sorted order
    float4* sx[2] = {nullptr, nullptr};
    int last_x = 0;
    float4* sv = nullptr;
    float4* sx0 = nullptr;
    float4* somega = nullptr;
    float4* dpb = nullptr;     // lambda-independent part of each delta-p sum (DevParams::dpb)
    float* rho = nullptr;
    uint32_t* lod = nullptr;
    // contacts
    float4* cand = nullptr;
    uint32_t* ct_counts = nullptr;
    uint32_t* scalars = nullptr;  // [0] contact count, [1] NaN count
    uint32_t contact_count_host = 0;
    bool contacts_valid = false;

    // SDF grid (active collision field)
    float* grid = nullptr;
    size_t grid_elems = 0;
    float* slab_min = nullptr;
    int dims[3] = {0, 0, 0};
    float origin[3] = {0, 0, 0};
    double origin_d[3] = {0, 0, 0};
    float cell = 0.0f;
    double cell_d = 0.0;
    bool sdf_attached = false;        // this handle owns a usable grid
    uint64_t grid_generation = 0;     // bumped whenever `grid` is reallocated
    // the SDF this fluid collides with: itself, another handle (borrowed,
    // like PBFluids::setSDFBoundary's non-owning pointer) or none
    pbf_handle* sdf_src = nullptr;
    uint64_t captured_generation = 0;
    float sdf_padding = 0.0f;
    bool sdf_containment = false;

    // triangle mesh + LBVH (pbf_mesh.cu)
    bool mesh_attached = false;
    pbf::MeshDev mesh{};
    void* mesh_host = nullptr;  // host-side build data
    long long* force_acc = nullptr;
    int* force_contacts = nullptr;
    float* force_out = nullptr;
    void mesh_free();

    // execution
    uint64_t launches = 0;
    bool use_graph = false;
    bool capturing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    uint64_t graph_launches = 0;

    // profiling
    struct ProfRec {
        int slot;
        cudaEvent_t a, b;
    };
    bool profiling = false;
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> event_pool;
    int prof_open[PBF_NUM_PASS_SLOTS];
    double prof_ms[PBF_NUM_PASS_SLOTS] = {};
    uint64_t prof_count[PBF_NUM_PASS_SLOTS] = {};

    ~pbf_handle();
    pbf::DevParams dev_params() const;
    pbf::SdfDev sdf_dev() const;
    int ensure_capacity(uint32_t need_n);
    void invalidate_graph();
    int upload_grid(const float* dist_host, const int32_t d[3], const float o[3], float c);
    int stage(int st, uint32_t iter);
    int step_body();
    int step();
    cudaEvent_t take_event();
    void prof_begin(int slot);
    void prof_end(int slot);
    int prof_collect();
};
