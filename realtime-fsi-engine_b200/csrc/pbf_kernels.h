// pbf_kernels.h — host-side launchers of the engine's kernels.
#pragma once

#include "pbf_internal.cuh"

namespace pbf {

// ---- k_solver.cu ------------------------------------------------------------
void launch_predict_hash(const DevParams& P, const float4* pos, const float4* vel, uint32_t* keys, int sms,
                         cudaStream_t st);
// `order` (may be null) lists sorted slots in the order threads take them:
// the 24-bit Morton order of the predict-time cells, so that the threads of a
// block share their neighbour buckets in L1.
void launch_reorder(const DevParams& P, const uint32_t* ids, const float4* pos, const float4* vel, float4* sx,
                    float4* sv, float4* sx0, uint32_t* lod, uint32_t* mcode, int sms, cudaStream_t st);
void launch_build_table(uint32_t n, const uint32_t* sk, int2* table, int sms, cudaStream_t st);
void launch_check_finite(uint32_t n, const float4* pos, const float4* vel, uint32_t* bad, int sms,
                         cudaStream_t st);
void launch_unpack_particles(uint32_t n, const float4* aos, float4* pos, float4* pred, float4* vel, int sms,
                             cudaStream_t st);
void launch_pack_particles(uint32_t n, const float4* pos, const float4* pred, const float4* vel, float4* aos,
                           int sms, cudaStream_t st);

// ---- k_masked.cu: thread per particle, bucket chunks tested into a hit mask --
void launch_lambda_m(const DevParams& P, const float4* xin, float4* xout, float* rho, const int2* table,
                     const uint32_t* lod, uint32_t iter, const uint32_t* order, cudaStream_t st);
void launch_deltap_m(const DevParams& P, const float4* xin, float4* xout, const int2* table, const uint32_t* lod,
                     uint32_t iter, const uint32_t* order, cudaStream_t st);
void launch_integrate_m(const DevParams& P, const float4* xs, const float4* sv, float4* sx0, float4* somega,
                        const uint32_t* ids, float4* pos, float4* vel, const int2* table, const uint32_t* order,
                        cudaStream_t st);
void launch_vorticity_m(const DevParams& P, const float4* spos, const float4* somega, const uint32_t* ids,
                        float4* vel, const int2* table, const uint32_t* order, cudaStream_t st);

// ---- k_dense.cu: x-runs of a dense cell window over relabelled data ----------
constexpr int kDenseListWords = 16;
// Label-space position/velocity arrays hold this many entries past the last
// label, so a run's last chunk of candidates may load past the run's end.
constexpr int kLabelPad = 32;
// Cells of margin around the walls' box in a dense window: they also hold the
// predict-time cells of particles that move towards a wall (x* = x + v dt lies
// beyond it until the walls clamp it).
constexpr int kDenseMargin = 6;
struct SceneDev;  // pbf_batch.h
// A dense window per scene: one scene (scenes == null), or the scenes of a
// batch, scene k's window occupying global slots [slot0_k, slot0_k + its
// cells).  The window fields below describe one window; the passes of a batch
// replace them, the hash mask, walls and SDF with the scene of each label.
struct DenseArgs {
    const int2* table;     // per window slot: label range of its particles, (-1, -1) when empty
    const int2* runs;      // per window slot: label range of slots s-1 .. s+1 of its row
    const uint32_t* order; // pass thread i takes label order[i] (null: label i)
    uint32_t* hm;          // lambda hit masks for the delta-p of the same iteration (kDenseListWords x n)
    uint8_t* hcnt;         // per label: chunks recorded, 0xFF = none
    int use_list;          // delta-p: the lambda pass of this iteration recorded hm/hcnt
    int rec_list;          // integrate: record hm/hcnt for the vorticity pass (positions it leaves in place)
    uint8_t* vmark;        // per window slot: a query there sees a particle integrate moved (no replay)
    uint32_t* rec_slot;    // delta-p / integrate (may be null): current slot of each output position
    uint32_t* rec_cnt;     //   and per-slot counts (zeroed by the caller), for the next pass's order
    const uint16_t* clean; // per window slot: rows (bit (dz+1)*3+(dy+1)) whose buckets a hash collision near the cell
                           //   affects; 0 = none, 0x1FF at the window's edge
    const uint8_t* dcol;   // per window slot: Chebyshev distance to the nearest other cell of its bucket
    uint32_t* dirty;       // per window slot: rows through whose buckets a moved particle with a colliding cell near
                           //   is within reach (same bits as `clean`)
    const int2* htable;    // the hashed cell table (sorted slots)
    const uint32_t* inv;   // hash slot -> label
    const float4* xb;      // predict-time x*, label order
    uint32_t* flag;        // [0] moved particles that marked cells this substep, [1] bucket walks
    int gx0, gy0, gz0;     // cell coordinates of window slot (0, 0, 0)
    uint32_t nx, ny, nz;   // window extent in cells
    float drift2;          // squared drift bound (0.9 h)^2
    uint32_t slot0;        // global slot of window slot (0, 0, 0)
    uint32_t total;        // slots of all windows (the thread order's extra slot is `total`)
    const SceneDev* scenes;      // batch: per-scene constants (null: one scene)
    const uint16_t* scene_of;    // batch: scene of each label / hash-sorted index (scene-contiguous)
    const uint16_t* slot_scene;  // batch: scene of each global slot
};
// The keys and the label-order gather straight from (pos, vel) of the
// hash-sorted ids, re-deriving x* and v' as the predict pass does.
void launch_d_keys_pred(const DevParams& P, const DenseArgs& D, const uint32_t* ids, const float4* pos,
                        const float4* vel, uint32_t* dkey, int sms, cudaStream_t st);
// One scene: the predict pass writing the hash keys and, for each particle,
// its predict-time window slot; the relabelling then gathers those slots.
void launch_d_predict_hash(const DevParams& P, const DenseArgs& D, const float4* pos, const float4* vel,
                           uint32_t* keys, uint32_t* dkey_id, int sms, cudaStream_t st);
void launch_d_keys_gather(uint32_t n, const uint32_t* ids, const uint32_t* dkey_id, uint32_t* dkey, int sms,
                          cudaStream_t st);
void launch_d_permute(const DevParams& P, const uint32_t* order, const uint32_t* ids, const uint32_t* skeys,
                      const float4* pos, const float4* vel, float4* lx, float4* lxb, float4* lv, float4* lx0,
                      uint32_t* lid, uint32_t* lkey, uint32_t* inv, int sms, cudaStream_t st);
void launch_d_clean(const DenseArgs& D, uint32_t mask, uint16_t* clean, uint32_t* unclean, int sms, cudaStream_t st);
void launch_d_dcol(const DenseArgs& D, uint32_t mask, uint8_t* dcol, int sms, cudaStream_t st);
void launch_d_runs(const DenseArgs& D, const int2* cells, int2* runs, int sms, cudaStream_t st);
// Labels bucketed by the window slot of their current cell (X) into order[n].
// Scratch: slot_of[n], cnt[slots + 1], block_sums[order_scan_blocks(slots)].
uint32_t order_scan_blocks(uint32_t slots);
void launch_d_order(const DevParams& P, const DenseArgs& D, const float4* X, uint32_t* slot_of, uint32_t* cnt,
                    uint32_t* block_sums, uint32_t* order, cudaStream_t st, uint64_t* launches);
// One scene's relabelling: for the hash-sorted sequence of slot keys dkey[n]
// (window slots, `slots` for the overflow) with hash keys skeys[n], order[t]
// = hash-sorted index of label t and sorted_keys[t] its key, as a stable sort
// by key orders them (the overflow slot's entries in any order).  Scratch:
// cnt[slots + 1], block_sums[order_scan_blocks(slots)], one overflow counter.
void launch_d_relabel(uint32_t n, uint32_t slots, const uint32_t* dkey, const uint32_t* skeys, uint32_t* cnt,
                      uint32_t* block_sums, uint32_t* overflow_count, uint32_t* order, uint32_t* sorted_keys, int sms,
                      cudaStream_t st, uint64_t* launches);
// The same order from slots and counts a pass recorded (DenseArgs::rec_slot / rec_cnt).
void launch_d_order_recorded(const DevParams& P, const DenseArgs& D, const uint32_t* slot_of, uint32_t* cnt,
                             uint32_t* block_sums, uint32_t* order, cudaStream_t st, uint64_t* launches);
void launch_d_lambda(const DevParams& P, const DenseArgs& D, const float4* lx_in, float4* lx_out, float* lrho,
                     cudaStream_t st);
void launch_d_deltap(const DevParams& P, const DenseArgs& D, const float4* lx_in, float4* lx_out, cudaStream_t st);
void launch_d_integrate(const DevParams& P, const DenseArgs& D, const float4* lx, const float4* lv, float4* lx0,
                        float4* lom, const uint32_t* lid, float4* pos, float4* vel, cudaStream_t st);
void launch_d_vorticity(const DevParams& P, const DenseArgs& D, const float4* lx0, const float4* lom,
                        const uint32_t* lid, float4* vel, cudaStream_t st);
void launch_d_unpermute4(uint32_t n, const uint32_t* inv, const float4* src, float4* dst, int sms, cudaStream_t st);
void launch_d_unpermute1(uint32_t n, const uint32_t* inv, const float* src, float* dst, int sms, cudaStream_t st);

// ---- k_sort.cu ----------------------------------------------------------------
// Keys per sort tile: one 256-digit histogram per tile, so scratch sized for
// n keys holds 256 * sort_num_tiles(n) histogram words.
constexpr uint32_t kSortTileKeys = 2048;
uint32_t sort_num_tiles(uint32_t n);
void launch_radix_sort(uint32_t n, uint32_t key_bits, const uint32_t* keys_in, uint32_t* ka, uint32_t* ia,
                       uint32_t* kb, uint32_t* ib, uint32_t* hist, uint32_t* totals, uint32_t** out_keys,
                       uint32_t** out_ids, cudaStream_t st, uint64_t* launches);
void launch_radix_sort_into(uint32_t n, uint32_t key_bits, const uint32_t* keys_in, uint32_t* out_k, uint32_t* out_i,
                            uint32_t* tmp_k, uint32_t* tmp_i, uint32_t* hist, uint32_t* totals, cudaStream_t st);

// ---- k_sdf.cu -----------------------------------------------------------------
void launch_sdf_slab_min(const float* dist, int dx, int dy, int dz, float* slab_min, cudaStream_t st);
void launch_sdf_sample(SdfDev S, const float* pts3, uint32_t n, float* d, float* grad3, cudaStream_t st);
// Contact compaction |sdf(pos)| < band in particle order.  Scratch: counts of
// contact_num_blocks(n) uint32 and one uint32 total.
uint32_t contact_num_blocks(uint32_t n);
void launch_contact_filter(SdfDev S, uint32_t n, const float4* pos, const float4* vel, float band,
                           uint32_t* block_counts, uint32_t* total, float4* out_cand, cudaStream_t st,
                           uint64_t* launches);

// ---- k_mesh.cu ------------------------------------------------------------------
struct MeshDev {
    int nv, nf;
    const int3* faces;    // nf
    float3* verts;        // nv, current positions
    float3* face_n;       // nf, refreshed on refit
    const float3* edge_n; // nf*3 (AB, AC, BC), build-time
    const float3* vert_n; // nv, build-time
    // LBVH over the faces (Karras 2012): nf leaves, nf-1 internal nodes
    int2* child;          // internal child indices; >= nf-1 + leaf marks leaves (encoded)
    int* parent;          // 2nf-1
    float4* bmin;         // 2nf-1 (xyz)
    float4* bmax;         // 2nf-1
    int* leaf_face;       // nf: face index of leaf i (Morton order)
    uint32_t* flags;      // nf-1 refit arrival counters
    const int* frontier;  // kMeshFrontier subtree roots that together cover the tree (-1: unused)
};
constexpr int kMeshFrontier = 32;  // one per lane of the grid kernel's warp
void launch_mesh_refit(MeshDev M, cudaStream_t st, uint64_t* launches);
// Vertex (angle-weighted) and edge pseudo-normals from M.face_n (run after
// launch_mesh_refit).  voff/vfc: per-vertex (face, corner) lists in face
// order; partner: per face edge slot (AB, AC, BC) the other face of an edge
// shared by exactly two faces, else -1.
void launch_mesh_pseudo_normals(MeshDev M, const int* voff, const int2* vfc, const int* partner, float3* vert_n,
                                float3* edge_n, cudaStream_t st, uint64_t* launches);
void launch_mesh_grid_d(MeshDev M, int dx, int dy, int dz, const double* origin, double cell, float* out, int sms,
                        cudaStream_t st);
void launch_morton(int nf, const int3* faces, const float3* verts, float3 lo, float3 inv_ext, uint32_t* codes,
                   cudaStream_t st);
void launch_mesh_closest(MeshDev M, const float* pts3, uint32_t n, int* face, float* point3, cudaStream_t st);
// Per-vertex force accumulation in 2^-32 fixed point (deterministic).
void launch_vertex_forces(MeshDev M, const float4* cand, const uint32_t* count, uint32_t cap, float band,
                          int use_vel, long long* acc3, int* contacts, cudaStream_t st);
void launch_forces_to_float(int nv, const long long* acc3, float* out3, cudaStream_t st);
// LBVH topology from sorted Morton codes (device).
void launch_lbvh_topology(int nf, const uint32_t* sorted_codes, int2* child, int* parent, cudaStream_t st);

}  // namespace pbf
