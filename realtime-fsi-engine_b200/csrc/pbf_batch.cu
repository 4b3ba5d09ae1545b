// pbf_batch.cu — the multi-scene engine of the pbf_batch_* C ABI.
//
// Step pipeline (one launch per pass for all scenes, replayed from a graph):
//   for each substep:
//     predict+offset hash -> radix sort of the offset keys (segmented by
//     construction) -> clear + fill the shared cell table -> reorder into
//     sorted float4 SoA (+ scene-prefixed Morton codes, sorted into the
//     processing order) -> I x (lambda, deltaP+apply) -> integrate
//   vorticity confinement (once per step)
// exactly the schedule of PBFluids::step (src/fluid/PBFluids.cpp:323-517)
// that the single-scene handle issues.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "../../include/pbf_b200.h"
#include "pbf_batch.h"
#include "pbf_engine.h"

using namespace pbf;

#define BCK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

#define CHECK_BATCH(b)                                                                             \
    do {                                                                                           \
        if (!(b)) return pbf::set_error(PBF_ERR_INVALID, "null batch");                            \
        cudaError_t e_ = cudaSetDevice((b)->device);                                               \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_));      \
    } while (0)

template <class T>
static int balloc(T*& p, size_t count)
{
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) return PBF_OK;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        return set_error(PBF_ERR_ALLOC, "cudaMalloc(%zu B): %s", count * sizeof(T), cudaGetErrorString(e));
    }
    return PBF_OK;
}

template <class T>
static void bfree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

static uint32_t ceil_log2(uint64_t v)
{
    uint32_t b = 0;
    while ((1ull << b) < v) ++b;
    return b;
}

pbf_batch::~pbf_batch()
{
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    invalidate_graph();
    for (auto& s : scenes) {
        bfree(s.grid);
        bfree(s.slab_min);
    }
    bfree(pos); bfree(vel); bfree(pred); bfree(aos); bfree(scene_of); bfree(scenes_dev);
    bfree(keys); bfree(ka); bfree(ia); bfree(kb); bfree(ib); bfree(hist); bfree(totals); bfree(table);
    bfree(mcode); bfree(mka); bfree(mia); bfree(mkb); bfree(mib);
    bfree(sx[0]); bfree(sx[1]); bfree(sv); bfree(sx0); bfree(somega); bfree(dpb); bfree(rho); bfree(lod);
    bfree(save_pos); bfree(save_vel);
    dense_free();
    ad_free();
    if (stream) cudaStreamDestroy(stream);
}

void pbf_batch::invalidate_graph()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    if (rec_exec) cudaGraphExecDestroy(rec_exec);
    if (rec_graph) cudaGraphDestroy(rec_graph);
    if (bwd_exec) cudaGraphExecDestroy(bwd_exec);
    if (bwd_graph) cudaGraphDestroy(bwd_graph);
    rec_exec = bwd_exec = nullptr;
    rec_graph = bwd_graph = nullptr;
}

// Shared constants; the walls, hash mask and SDF of DevParams are unused
// here (per scene in SceneDev).
DevParams pbf_batch::dev_params() const
{
    DevParams P;
    std::memset(&P, 0, sizeof(P));
    for (int a = 0; a < 3; ++a) {
        P.bmin[a] = derived.bounds_min[a];
        P.bmax[a] = derived.bounds_max[a];
        P.g[a] = derived.gravity_dt[a];
    }
    P.dt = derived.gravity_dt[3];
    P.inv_dt = (P.dt > 0.0f) ? 1.0f / P.dt : 0.0f;
    P.h = derived.h;
    P.h2 = derived.h * derived.h;
    P.rho0 = derived.rho0;
    P.inv_rho0 = derived.inv_rho0;
    P.inv_rho0_sq = derived.inv_rho0 * derived.inv_rho0;
    P.eps = derived.eps;
    P.wq = derived.wq;
    P.inv_wq = derived.wq > 0.0f ? 1.0f / derived.wq : 0.0f;
    P.k_corr = derived.k_corr;
    P.n_corr = derived.n_corr;
    P.ncorr_is4 = derived.n_corr == 4.0f ? 1u : 0u;
    P.viscosity = derived.viscosity;
    P.damping = derived.bound_damping;
    P.cohesion = derived.cohesion_strength;
    P.w0_self = derived.w0_self;
    P.poly6 = derived.poly6_coeff;
    P.spiky = derived.spiky_coeff;
    P.max_dp = 0.5f * derived.h;
    P.mask = derived.hash_mask;
    P.n = n;
    P.scorr = derived.enable_scorr;
    P.visc_on = derived.enable_viscosity;
    P.vort_on = cfg.enable_vorticity ? 1u : 0u;
    P.apbf = derived.enable_apbf;
    P.vort_eps = cfg.vorticity_epsilon;
    P.interacting = 0u;
    P.i_radius = derived.interaction_radius;
    P.i_strength = derived.interaction_strength;
    P.lod_max_dist = derived.lod_max_dist;
    P.min_lod = derived.min_lod;
    P.max_lod = derived.max_lod;
    P.dpb = dpb;
    return P;
}

// Per-scene constants to the device: walls with padding (PBFluids::setBounds,
// PBFluids.cpp:299-306), bucket offsets, Morton origins and SDF descriptors.
int pbf_batch::upload_scenes()
{
    std::vector<SceneDev> hs(scenes.size());
    const float h = cfg.h;
    uint32_t max_span = 1;
    for (size_t k = 0; k < scenes.size(); ++k) {
        const Scene& s = scenes[k];
        SceneDev& d = hs[k];
        std::memset(&d, 0, sizeof(d));
        d.table_off = s.table_off;
        d.mask = s.desc.hash_size - 1u;
        for (int a = 0; a < 3; ++a) {
            d.bmin[a] = s.desc.bounds_min[a] + collision_padding;
            d.bmax[a] = s.desc.bounds_max[a] - collision_padding;
            const int lo = (int)std::floor(s.desc.bounds_min[a] / h) - 1;
            const int hi = (int)std::floor(s.desc.bounds_max[a] / h) + 1;
            d.cell_lo[a] = lo;
            max_span = std::max(max_span, (uint32_t)std::max(hi - lo + 1, 1));
        }
        if (s.sdf_on && s.grid) {
            d.sdf.dist = s.grid;
            d.sdf.slab_min = s.slab_min;
            d.sdf.dx = s.dims[0];
            d.sdf.dy = s.dims[1];
            d.sdf.dz = s.dims[2];
            d.sdf.ox = s.origin[0] + s.sdf_offset[0];
            d.sdf.oy = s.origin[1] + s.sdf_offset[1];
            d.sdf.oz = s.origin[2] + s.sdf_offset[2];
            d.sdf.cell = s.cell;
            d.sdf.inv_cell = 1.0f / s.cell;
            d.sdf.padding = s.sdf_padding;
            d.sdf.containment = s.containment ? 1 : 0;
            d.sdf.enabled = 1;
        }
    }
    // Morton bits per axis: enough for the widest scene, the scene index
    // above them, within 32 bits (wider scenes wrap, which only costs
    // locality).
    // dense windows (neighbour mode 8): each scene's walls in cells, as the
    // kernels compute a cell, with kDenseMargin cells of margin (the
    // single-scene window), one after another in the global slot space
    std::vector<int> w(7 * scenes.size());
    uint64_t total = 0;
    bool fits = true;
    for (size_t k = 0; k < scenes.size(); ++k) {
        SceneDev& d = hs[k];
        uint64_t cells = 1;
        for (int a = 0; a < 3; ++a) {
            const float lo = std::floor(d.bmin[a] / h), hi = std::floor(d.bmax[a] / h);
            const bool ok = lo >= -1e7f && hi <= 1e7f && hi >= lo && hi - lo < 1e6f;
            fits = fits && ok;
            d.win_g0[a] = ok ? (int)lo - kDenseMargin : 0;
            d.win_n[a] = ok ? (uint32_t)((int)hi - (int)lo + 1 + 2 * kDenseMargin) : 1u;
            cells *= d.win_n[a];
        }
        d.slot0 = (uint32_t)std::min<uint64_t>(total, 0xFFFFFFFFull);
        total = std::min<uint64_t>(total + cells, 1ull << 40);
        for (int a = 0; a < 3; ++a) {
            w[7 * k + a] = d.win_g0[a];
            w[7 * k + 3 + a] = (int)d.win_n[a];
        }
        w[7 * k + 6] = (int)d.slot0;
    }
    if (!fits) total = 1ull << 40;  // no dense windows (dense_fits() is false)
    if (w != win || total != dense_total) dense_ready = false;
    win = w;
    dense_total = total;
    const uint32_t sbits = ceil_log2(scenes.size());
    mbits = std::min<uint32_t>(std::max<uint32_t>(ceil_log2(max_span), 1u), 10u);
    while (sbits + 3 * mbits > 32) --mbits;
    order_bits = sbits + 3 * mbits;
    BCK(cudaMemcpyAsync(scenes_dev, hs.data(), sizeof(SceneDev) * hs.size(), cudaMemcpyHostToDevice, stream));
    BCK(cudaStreamSynchronize(stream));
    invalidate_graph();
    return PBF_OK;
}

// One substep from (src_pos, src_vel) to (dst_pos, dst_vel); the sorted
// arrays, table and processing order are left describing this substep.
int pbf_batch::substep_body(const float4* src_pos, const float4* src_vel, float4* dst_pos, float4* dst_vel)
{
    const DevParams P = dev_params();
    const int sms = num_sms;
    BatchLaunch L = launch;
    L.sms = sms;
    const uint32_t max_iter = derived.enable_apbf ? derived.max_lod : cfg.solver_iterations;
    launch_b_predict(P, scenes_dev, scene_of, src_pos, src_vel, keys, sms, stream);
    launch_radix_sort(n, key_bits, keys, ka, ia, kb, ib, hist, totals, &skeys, &ids, stream, &launches);
    BCK(cudaMemsetAsync(table, 0xFF, sizeof(int2) * (size_t)table_size, stream));
    launch_build_table(n, skeys, table, sms, stream);
    launch_b_reorder(P, scenes_dev, scene_of, ids, src_pos, src_vel, sx[0], sv, sx0, lod, morton ? mcode : nullptr,
                     mbits, sms, stream);
    launches += 3;
    order = nullptr;
    if (morton) {
        uint32_t* msorted = nullptr;
        launch_radix_sort(n, order_bits, mcode, mka, mia, mkb, mib, hist, totals, &msorted, &order, stream,
                          &launches);
    }
    for (uint32_t it = 1; it <= max_iter; ++it) {
        launch_b_lambda(P, L, scenes_dev, scene_of, sx[0], sx[1], rho, table, lod, it, order, stream);
        launch_b_deltap(P, L, scenes_dev, scene_of, sx[1], sx[0], table, lod, it, order, stream);
        launches += 2;
    }
    launch_b_integrate(P, L, scenes_dev, scene_of, sx[0], sv, sx0, somega, ids, dst_pos, dst_vel, table, order,
                       stream);
    ++launches;
    return PBF_OK;
}

int pbf_batch::effective_mode() const
{
    if (neighbour_mode == 4 || neighbour_mode == 8) return neighbour_mode;
    if (tuned_mode) return tuned_mode;
    return dense_fits() && n >= (1u << 19) ? 8 : 4;
}

void pbf_batch::dense_free()
{
    bfree(lx[0]); bfree(lx[1]); bfree(lxb); bfree(lv); bfree(lx0); bfree(lom); bfree(lrho);
    bfree(lid); bfree(lkey); bfree(inv); bfree(dtable); bfree(druns); bfree(dclean); bfree(ddcol);
    bfree(ddirty); bfree(dhcnt); bfree(dvmark); bfree(dslot_scene); bfree(dflag); bfree(dslot); bfree(dord); bfree(dcnt);
    bfree(dbsum); bfree(dhm);
    dense_ready = false;
}

// Buffers of mode 8 and the per-slot tables that depend only on the windows
// and hash masks (conditions (a), (b) and the colliding-cell distance of
// k_dense.cu); called outside graph capture whenever the windows changed.
int pbf_batch::dense_setup()
{
    if (!dense_fits())
        return set_error(PBF_ERR_INVALID, "dense windows need %llu slots (at most 2^26) and APBF off",
                         (unsigned long long)dense_total);
    if (capturing) return set_error(PBF_ERR_STATE, "dense windows changed during graph capture");
    int rc;
    const size_t c = std::max<uint32_t>(n, 1u), cp = c + kLabelPad, T = (size_t)dense_total;
    if (!lx[0]) {
        if ((rc = balloc(lx[0], cp)) || (rc = balloc(lx[1], cp)) || (rc = balloc(lxb, c)) || (rc = balloc(lv, cp)) ||
            (rc = balloc(lx0, cp)) || (rc = balloc(lom, cp)) || (rc = balloc(lrho, c)) || (rc = balloc(lid, c)) ||
            (rc = balloc(lkey, c)) || (rc = balloc(inv, c)) || (rc = balloc(dslot, c)) || (rc = balloc(dord, c)) ||
            (rc = balloc(dhm, c * kDenseListWords)) || (rc = balloc(dhcnt, c)) || (rc = balloc(dflag, 4))) {
            dense_free();
            return rc;
        }
    }
    if ((rc = balloc(dtable, T)) || (rc = balloc(druns, T)) || (rc = balloc(dclean, T)) || (rc = balloc(ddcol, T)) ||
        (rc = balloc(ddirty, T)) || (rc = balloc(dvmark, T)) || (rc = balloc(dslot_scene, T)) || (rc = balloc(dcnt, T + 1)) ||
        (rc = balloc(dbsum, order_scan_blocks((uint32_t)T)))) {
        dense_free();
        return rc;
    }
    std::vector<uint16_t> ss(T);
    for (size_t k = 0; k < scenes.size(); ++k) {
        const size_t b0 = (size_t)(uint32_t)win[7 * k + 6];
        const size_t cells = (size_t)win[7 * k + 3] * (size_t)win[7 * k + 4] * (size_t)win[7 * k + 5];
        std::fill(ss.begin() + b0, ss.begin() + b0 + cells, (uint16_t)k);
    }
    BCK(cudaMemcpyAsync(dslot_scene, ss.data(), sizeof(uint16_t) * T, cudaMemcpyHostToDevice, stream));
    BCK(cudaMemsetAsync(dflag, 0, sizeof(uint32_t) * 4, stream));
    const DenseArgs D = dense_args();
    launch_d_clean(D, 0u, dclean, dflag + 2, num_sms, stream);
    launch_d_dcol(D, 0u, ddcol, num_sms, stream);
    launches += 2;
    BCK(cudaStreamSynchronize(stream));
    BCK(cudaGetLastError());
    dense_ready = true;
    return PBF_OK;
}

DenseArgs pbf_batch::dense_args() const
{
    DenseArgs D;
    std::memset(&D, 0, sizeof(D));
    D.table = dtable;
    D.runs = druns;
    D.hm = dhm;
    D.hcnt = dhcnt;
    D.clean = dclean;
    D.dcol = ddcol;
    D.dirty = ddirty;
    D.vmark = dvmark;
    D.htable = table;
    D.inv = inv;
    D.xb = lxb;
    D.flag = dflag;
    const float b = 0.9f * derived.h;
    D.drift2 = b * b;
    D.total = (uint32_t)dense_total;
    D.scenes = scenes_dev;
    D.scene_of = scene_of;
    D.slot_scene = dslot_scene;
    return D;
}

// The step in mode 8: per substep the hashed sort and table (the walk of
// particles that fail the window conditions), the relabelling by global window
// slot, then the passes of k_dense.cu over all scenes at once.  Passes after
// the first iteration take their threads in current-cell order from the
// slots the previous pass recorded; delta-p replays its lambda's hit masks.
int pbf_batch::dense_step_body()
{
    const DevParams P = dev_params();
    const int sms = num_sms;
    const uint32_t T = (uint32_t)dense_total;
    const uint32_t slot_bits = std::max<uint32_t>(ceil_log2(T), 1u);
    const uint32_t iters = cfg.solver_iterations;
    const bool vort = cfg.enable_vorticity;
    DenseArgs D = dense_args();
    auto record = [&]() -> int {
        BCK(cudaMemsetAsync(dcnt, 0, sizeof(uint32_t) * ((size_t)T + 1), stream));
        D.rec_slot = dslot;
        D.rec_cnt = dcnt;
        return PBF_OK;
    };
    auto order_recorded = [&]() {
        launch_d_order_recorded(P, D, dslot, dcnt, dbsum, dord, stream, &launches);
        D.order = dord;
    };
    for (uint32_t sub = 0; sub < cfg.substep_iterations; ++sub) {
        const bool last = sub + 1 == cfg.substep_iterations;
        launch_b_predict(P, scenes_dev, scene_of, pos, vel, keys, sms, stream);
        launch_radix_sort(n, key_bits, keys, ka, ia, kb, ib, hist, totals, &skeys, &ids, stream, &launches);
        BCK(cudaMemsetAsync(table, 0xFF, sizeof(int2) * (size_t)table_size, stream));
        launch_build_table(n, skeys, table, sms, stream);
        D = dense_args();
        launch_d_keys_pred(P, D, ids, pos, vel, mcode, sms, stream);
        launches += 3;
        uint32_t *msorted = nullptr, *lorder = nullptr;
        launch_radix_sort(n, slot_bits, mcode, mka, mia, mkb, mib, hist, totals, &msorted, &lorder, stream,
                          &launches);
        launch_d_permute(P, lorder, ids, skeys, pos, vel, lx[0], lxb, lv, lx0, lid, lkey, inv, sms, stream);
        BCK(cudaMemsetAsync(dtable, 0xFF, sizeof(int2) * (size_t)T, stream));
        launch_build_table(n, msorted, dtable, sms, stream);
        launch_d_runs(D, dtable, druns, sms, stream);
        BCK(cudaMemsetAsync(ddirty, 0, sizeof(uint32_t) * (size_t)T, stream));
        BCK(cudaMemsetAsync(dflag, 0, sizeof(uint32_t), stream));
        launches += 3;
        for (uint32_t it = 1; it <= iters; ++it) {
            D.rec_slot = nullptr;
            D.rec_cnt = nullptr;
            D.use_list = 0;
            if (it >= 2) order_recorded();
            launch_d_lambda(P, D, lx[0], lx[1], lrho, stream);
            D.use_list = 1;
            if (const int rc = record()) return rc;
            launch_d_deltap(P, D, lx[1], lx[0], stream);
            launches += 2;
        }
        D.rec_slot = nullptr;
        D.rec_cnt = nullptr;
        D.use_list = 0;
        order_recorded();
        if (last && vort) {
            if (const int rc = record()) return rc;
            // hit masks for the vorticity pass
            BCK(cudaMemsetAsync(dvmark, 0, (size_t)T, stream));
            D.rec_list = 1;
        }
        launch_d_integrate(P, D, lx[0], lv, lx0, lom, lid, pos, vel, stream);
        D.rec_list = 0;
        ++launches;
    }
    if (vort) {
        D.rec_slot = nullptr;
        D.rec_cnt = nullptr;
        D.use_list = 1;
        order_recorded();
        launch_d_vorticity(P, D, lx0, lom, lid, vel, stream);
        ++launches;
    }
    return PBF_OK;
}

int pbf_batch::step_body()
{
    if (effective_mode() == 8) return dense_step_body();
    const DevParams P = dev_params();
    BatchLaunch L = launch;
    L.sms = num_sms;
    for (uint32_t sub = 0; sub < cfg.substep_iterations; ++sub) {
        const int rc = substep_body(pos, vel, pos, vel);
        if (rc) return rc;
    }
    if (cfg.enable_vorticity) {
        launch_b_vorticity(P, L, scenes_dev, scene_of, sx0, somega, ids, vel, table, order, stream);
        ++launches;
    }
    return PBF_OK;
}

int pbf_batch::step()
{
    if (n == 0) return PBF_OK;
    if (effective_mode() == 8 && !dense_ready) {
        invalidate_graph();
        if (const int rc = dense_setup()) return rc;
    }
    if (use_graph) {
        if (!graph_exec) {
            const uint64_t before = launches;
            capturing = true;
            BCK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            const int rc = step_body();
            cudaGraph_t g = nullptr;
            const cudaError_t e = cudaStreamEndCapture(stream, &g);
            capturing = false;
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
            graph = g;
            BCK(cudaGraphInstantiate(&graph_exec, graph, 0));
            graph_launches = launches - before;
            launches = before;
        }
        BCK(cudaGraphLaunch(graph_exec, stream));
        launches += graph_launches;
    } else {
        const int rc = step_body();
        if (rc) return rc;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return PBF_OK;
}

// ---- C ABI -----------------------------------------------------------------------------------
extern "C" int pbf_batch_create(const pbf_fluid_config* cfg, const pbf_scene_desc* descs, uint32_t num_scenes,
                                int device, pbf_batch** out)
{
    if (!out) return set_error(PBF_ERR_INVALID, "null output batch");
    *out = nullptr;
    if (!cfg || !descs) return set_error(PBF_ERR_INVALID, "null config or scenes");
    if (num_scenes == 0 || num_scenes > 65535u) return set_error(PBF_ERR_INVALID, "num_scenes %u not in [1, 65535]", num_scenes);
    pbf_derived_params probe;
    int rc = pbf_derive_params(cfg, 0.0f, &probe);
    if (rc) return rc;
    if (cfg->hash_size == 0 || (cfg->hash_size & (cfg->hash_size - 1u)) != 0)
        return set_error(PBF_ERR_INVALID, "hash_size %u is not a power of two", cfg->hash_size);
    if (cfg->substep_iterations == 0 || !(cfg->h > 0.0f) || !(cfg->rho0 > 0.0f))
        return set_error(PBF_ERR_INVALID, "invalid solver constants");
    uint64_t total = 0, table_total = 0;
    for (uint32_t k = 0; k < num_scenes; ++k) {
        const uint32_t hs = descs[k].hash_size ? descs[k].hash_size : cfg->hash_size;
        if ((hs & (hs - 1u)) != 0) return set_error(PBF_ERR_INVALID, "scene %u: hash_size %u is not a power of two", k, hs);
        total += descs[k].num_particles;
        table_total += hs;
    }
    if (total > (1ull << 31) || table_total > (1ull << 31))
        return set_error(PBF_ERR_INVALID, "batch too large (%llu particles, %llu buckets)",
                         (unsigned long long)total, (unsigned long long)table_total);
    int ndev = 0;
    BCK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return set_error(PBF_ERR_INVALID, "device %d out of range (%d)", device, ndev);
    BCK(cudaSetDevice(device));

    pbf_batch* b = new pbf_batch();
    b->device = device;
    b->cfg = *cfg;
    cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return set_error(PBF_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    b->scenes.resize(num_scenes);
    uint32_t off = 0, toff = 0;
    std::vector<uint16_t> sid((size_t)total);
    for (uint32_t k = 0; k < num_scenes; ++k) {
        pbf_batch::Scene& s = b->scenes[k];
        s.desc = descs[k];
        if (!s.desc.hash_size) s.desc.hash_size = cfg->hash_size;
        s.offset = off;
        s.table_off = toff;
        std::fill(sid.begin() + off, sid.begin() + off + s.desc.num_particles, (uint16_t)k);
        off += s.desc.num_particles;
        toff += s.desc.hash_size;
    }
    b->n = (uint32_t)total;
    b->table_size = (uint32_t)table_total;
    b->key_bits = std::max<uint32_t>(ceil_log2(table_total), 1u);
    b->cfg.particle_count = b->n;
    pbf_derive_params(&b->cfg, 0.0f, &b->derived);
    const size_t c = std::max<uint32_t>(b->n, 1u);
    if ((rc = balloc(b->pos, c)) || (rc = balloc(b->vel, c)) || (rc = balloc(b->pred, c)) ||
        (rc = balloc(b->aos, 3 * c)) || (rc = balloc(b->scene_of, c)) || (rc = balloc(b->scenes_dev, num_scenes)) ||
        (rc = balloc(b->keys, c)) || (rc = balloc(b->ka, c)) || (rc = balloc(b->ia, c)) || (rc = balloc(b->kb, c)) ||
        (rc = balloc(b->ib, c)) || (rc = balloc(b->hist, (size_t)256 * sort_num_tiles((uint32_t)c))) ||
        (rc = balloc(b->totals, 256)) || (rc = balloc(b->table, std::max<uint32_t>(b->table_size, 1u))) ||
        (rc = balloc(b->mcode, c)) || (rc = balloc(b->mka, c)) || (rc = balloc(b->mia, c)) ||
        (rc = balloc(b->mkb, c)) || (rc = balloc(b->mib, c)) || (rc = balloc(b->sx[0], c)) ||
        (rc = balloc(b->sx[1], c)) || (rc = balloc(b->sv, c)) || (rc = balloc(b->sx0, c)) ||
        (rc = balloc(b->somega, c)) || (rc = balloc(b->dpb, c)) || (rc = balloc(b->rho, c)) || (rc = balloc(b->lod, c))) {
        delete b;
        return rc;
    }
    cudaMemsetAsync(b->pos, 0, sizeof(float4) * c, b->stream);
    cudaMemsetAsync(b->vel, 0, sizeof(float4) * c, b->stream);
    cudaMemsetAsync(b->pred, 0, sizeof(float4) * c, b->stream);
    cudaMemsetAsync(b->somega, 0, sizeof(float4) * c, b->stream);
    cudaMemsetAsync(b->dpb, 0, sizeof(float4) * c, b->stream);
    if (total) cudaMemcpyAsync(b->scene_of, sid.data(), sizeof(uint16_t) * total, cudaMemcpyHostToDevice, b->stream);
    if ((rc = b->upload_scenes())) {
        delete b;
        return rc;
    }
    *out = b;
    return PBF_OK;
}

extern "C" int pbf_batch_destroy(pbf_batch* b)
{
    delete b;
    return PBF_OK;
}

extern "C" int pbf_batch_info(const pbf_batch* b, uint32_t* num_scenes, uint32_t* total)
{
    if (!b) return set_error(PBF_ERR_INVALID, "null batch");
    if (num_scenes) *num_scenes = (uint32_t)b->scenes.size();
    if (total) *total = b->n;
    return PBF_OK;
}

extern "C" int pbf_batch_scene_range(const pbf_batch* b, uint32_t scene, uint32_t* offset, uint32_t* count)
{
    if (!b) return set_error(PBF_ERR_INVALID, "null batch");
    if (scene >= b->scenes.size()) return set_error(PBF_ERR_INVALID, "scene %u out of range (%zu)", scene, b->scenes.size());
    if (offset) *offset = b->scenes[scene].offset;
    if (count) *count = b->scenes[scene].desc.num_particles;
    return PBF_OK;
}

extern "C" int pbf_batch_set_collision_padding(pbf_batch* b, float padding)
{
    CHECK_BATCH(b);
    b->collision_padding = padding;
    return b->upload_scenes();
}

// Range [off, off + cnt) addressed by `scene` (or all), validated against n.
static int batch_range(const pbf_batch* b, uint32_t scene, uint32_t n, uint32_t* off, uint32_t* cnt)
{
    if (scene == PBF_BATCH_ALL) {
        *off = 0;
        *cnt = b->n;
    } else {
        if (scene >= b->scenes.size())
            return set_error(PBF_ERR_INVALID, "scene %u out of range (%zu)", scene, b->scenes.size());
        *off = b->scenes[scene].offset;
        *cnt = b->scenes[scene].desc.num_particles;
    }
    if (n != *cnt) return set_error(PBF_ERR_INVALID, "scene holds %u particles, got n=%u", *cnt, n);
    return PBF_OK;
}

extern "C" int pbf_batch_set_particles(pbf_batch* b, uint32_t scene, const pbf_particle* ps, uint32_t n)
{
    CHECK_BATCH(b);
    uint32_t off = 0, cnt = 0;
    int rc = batch_range(b, scene, n, &off, &cnt);
    if (rc) return rc;
    if (cnt == 0) return PBF_OK;
    if (!ps) return set_error(PBF_ERR_INVALID, "null particles");
    BCK(cudaMemcpyAsync(b->aos + 3 * (size_t)off, ps, sizeof(pbf_particle) * (size_t)cnt, cudaMemcpyHostToDevice,
                        b->stream));
    launch_unpack_particles(cnt, b->aos + 3 * (size_t)off, b->pos + off, b->pred + off, b->vel + off, b->num_sms,
                            b->stream);
    ++b->launches;
    BCK(cudaStreamSynchronize(b->stream));
    return PBF_OK;
}

extern "C" int pbf_batch_read_particles(pbf_batch* b, uint32_t scene, pbf_particle* out, uint32_t n)
{
    CHECK_BATCH(b);
    uint32_t off = 0, cnt = 0;
    int rc = batch_range(b, scene, n, &off, &cnt);
    if (rc) return rc;
    if (cnt == 0) return PBF_OK;
    if (!out) return set_error(PBF_ERR_INVALID, "null output");
    launch_pack_particles(cnt, b->pos + off, b->pred + off, b->vel + off, b->aos + 3 * (size_t)off, b->num_sms,
                          b->stream);
    ++b->launches;
    BCK(cudaMemcpyAsync(out, b->aos + 3 * (size_t)off, sizeof(pbf_particle) * (size_t)cnt, cudaMemcpyDeviceToHost,
                        b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    return PBF_OK;
}

extern "C" int pbf_batch_set_sdf_grid(pbf_batch* b, uint32_t scene, const float* dist, const int32_t dims[3],
                                      const float origin[3], float cell)
{
    CHECK_BATCH(b);
    if (scene >= b->scenes.size()) return set_error(PBF_ERR_INVALID, "scene %u out of range", scene);
    if (!dist || !dims || !origin) return set_error(PBF_ERR_INVALID, "null argument");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return set_error(PBF_ERR_INVALID, "bad SDF dims");
    if ((size_t)dims[0] * dims[1] * dims[2] > (size_t)1 << 31) return set_error(PBF_ERR_INVALID, "SDF grid too large");
    if (!(cell > 0.0f)) return set_error(PBF_ERR_INVALID, "SDF cell size must be > 0");
    BCK(cudaStreamSynchronize(b->stream));
    pbf_batch::Scene& s = b->scenes[scene];
    const size_t total = (size_t)dims[0] * dims[1] * dims[2];
    const size_t have = (size_t)s.dims[0] * s.dims[1] * s.dims[2];
    int rc;
    if (!s.grid || total != have) {
        if ((rc = balloc(s.grid, total))) return rc;
    }
    if (!s.slab_min && (rc = balloc(s.slab_min, 6))) return rc;
    for (int a = 0; a < 3; ++a) {
        s.dims[a] = dims[a];
        s.origin[a] = origin[a];
    }
    s.cell = cell;
    BCK(cudaMemcpyAsync(s.grid, dist, total * sizeof(float), cudaMemcpyHostToDevice, b->stream));
    launch_sdf_slab_min(s.grid, dims[0], dims[1], dims[2], s.slab_min, b->stream);
    ++b->launches;
    s.sdf_on = true;
    return b->upload_scenes();
}

extern "C" int pbf_batch_set_sdf_mode(pbf_batch* b, uint32_t scene, float padding, uint32_t containment)
{
    CHECK_BATCH(b);
    if (scene >= b->scenes.size()) return set_error(PBF_ERR_INVALID, "scene %u out of range", scene);
    b->scenes[scene].sdf_padding = padding;
    b->scenes[scene].containment = containment != 0;
    return b->upload_scenes();
}

extern "C" int pbf_batch_clear_sdf(pbf_batch* b, uint32_t scene)
{
    CHECK_BATCH(b);
    if (scene >= b->scenes.size()) return set_error(PBF_ERR_INVALID, "scene %u out of range", scene);
    b->scenes[scene].sdf_on = false;
    return b->upload_scenes();
}

extern "C" int pbf_batch_step(pbf_batch* b)
{
    CHECK_BATCH(b);
    return b->step();
}

extern "C" int pbf_batch_sync(pbf_batch* b)
{
    CHECK_BATCH(b);
    BCK(cudaStreamSynchronize(b->stream));
    return PBF_OK;
}

extern "C" int pbf_batch_get_stream(pbf_batch* b, void** s)
{
    if (!b || !s) return set_error(PBF_ERR_INVALID, "null argument");
    *s = (void*)b->stream;
    return PBF_OK;
}

extern "C" int pbf_batch_device_ptrs(pbf_batch* b, void** pos4, void** vel4)
{
    if (!b) return set_error(PBF_ERR_INVALID, "null batch");
    if (pos4) *pos4 = (void*)b->pos;
    if (vel4) *vel4 = (void*)b->vel;
    return PBF_OK;
}

extern "C" int pbf_batch_kernel_launches(const pbf_batch* b, uint64_t* count)
{
    if (!b || !count) return set_error(PBF_ERR_INVALID, "null argument");
    *count = b->launches;
    return PBF_OK;
}

extern "C" int pbf_batch_set_option(pbf_batch* b, int option, int value)
{
    if (!b) return set_error(PBF_ERR_INVALID, "null batch");
    switch (option) {
    case PBF_BOPT_BLOCK:
        if (value != 64 && value != 128 && value != 256)
            return set_error(PBF_ERR_INVALID, "block size %d not in {64, 128, 256}", value);
        b->launch.block = value;
        break;
    case PBF_BOPT_ORDER:
        if (value != 0 && value != 1) return set_error(PBF_ERR_INVALID, "order %d not in {0, 1}", value);
        b->morton = value;
        break;
    case PBF_BOPT_BLOCKS_PER_SM:
        if (value < 0 || value > 64) return set_error(PBF_ERR_INVALID, "blocks per SM %d not in [0, 64]", value);
        b->launch.blocks_per_sm = value;
        break;
    case PBF_BOPT_USE_GRAPH:
        b->use_graph = value != 0;
        break;
    case PBF_BOPT_NEIGHBOUR_MODE:
        if (value != -1 && value != 4 && value != 8)
            return set_error(PBF_ERR_INVALID, "neighbour mode %d not in {-1, 4, 8}", value);
        if (value == 8 && !b->dense_fits())
            return set_error(PBF_ERR_INVALID, "dense windows need %llu slots (at most 2^26) and APBF off",
                             (unsigned long long)b->dense_total);
        b->neighbour_mode = value;
        b->tuned_mode = 0;
        break;
    default:
        return set_error(PBF_ERR_INVALID, "unknown batch option %d", option);
    }
    b->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_batch_get_option(const pbf_batch* b, int option, int* value)
{
    if (!b || !value) return set_error(PBF_ERR_INVALID, "null argument");
    switch (option) {
    case PBF_BOPT_BLOCK: *value = b->launch.block; break;
    case PBF_BOPT_ORDER: *value = b->morton; break;
    case PBF_BOPT_BLOCKS_PER_SM: *value = b->launch.blocks_per_sm; break;
    case PBF_BOPT_USE_GRAPH: *value = b->use_graph ? 1 : 0; break;
    case PBF_BOPT_NEIGHBOUR_MODE: *value = b->neighbour_mode; break;
    default: return set_error(PBF_ERR_INVALID, "unknown batch option %d", option);
    }
    return PBF_OK;
}

// Autotuner: every candidate (neighbour mode 8 when the windows fit; block x
// order x persistence in mode 4) is timed with CUDA events over `trial_steps`
// graph replays after one warm-up replay (which also captures the graph); the
// particle state is saved before and restored after, so tuning leaves the
// simulation where it was.
extern "C" int pbf_batch_autotune(pbf_batch* b, uint32_t trial_steps, pbf_batch_tuning* best,
                                  pbf_batch_tuning* results, uint32_t max_results, uint32_t* num_results)
{
    CHECK_BATCH(b);
    if (trial_steps == 0) return set_error(PBF_ERR_INVALID, "trial_steps must be >= 1");
    if (num_results) *num_results = 0;
    if (b->n == 0) return set_error(PBF_ERR_STATE, "empty batch");
    int rc = PBF_OK;
    const size_t c = b->n;
    if (!b->save_pos && (rc = balloc(b->save_pos, c))) return rc;
    if (!b->save_vel && (rc = balloc(b->save_vel, c))) return rc;
    BCK(cudaMemcpyAsync(b->save_pos, b->pos, sizeof(float4) * c, cudaMemcpyDeviceToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->save_vel, b->vel, sizeof(float4) * c, cudaMemcpyDeviceToDevice, b->stream));
    const bool graph_was = b->use_graph;
    b->use_graph = true;
    cudaEvent_t e0, e1;
    BCK(cudaEventCreate(&e0));
    BCK(cudaEventCreate(&e1));
    pbf_batch_tuning pick{b->launch.block, b->morton, b->launch.blocks_per_sm, 1e30f, 4};
    uint32_t count = 0;
    const int blocks[3] = {64, 128, 256};
    const int mode_was = b->neighbour_mode;
    auto time_steps = [&](float* ms) -> int {
        b->invalidate_graph();
        int r = b->step();
        if (r) return r;
        cudaEventRecord(e0, b->stream);
        for (uint32_t i = 0; i < trial_steps && !r; ++i) r = b->step();
        cudaEventRecord(e1, b->stream);
        if (r) return r;
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
        cudaEventElapsedTime(ms, e0, e1);
        *ms /= (float)trial_steps;
        return PBF_OK;
    };
    if (mode_was != 4 && b->dense_fits()) {
        b->neighbour_mode = 8;
        float ms = 0.0f;
        rc = time_steps(&ms);
        if (!rc) {
            const pbf_batch_tuning r{b->launch.block, b->morton, b->launch.blocks_per_sm, ms, 8};
            if (results && count < max_results) results[count] = r;
            ++count;
            pick = r;
        }
    }
    b->neighbour_mode = 4;
    for (int order = 0; order <= 1 && !rc && mode_was != 8; ++order) {
        for (int bi = 0; bi < 3 && !rc; ++bi) {
            const int occ = batch_max_blocks_per_sm(blocks[bi]);
            const int bps_list[2] = {0, occ};
            for (int pi = 0; pi < 2 && !rc; ++pi) {
                b->launch.block = blocks[bi];
                b->morton = order;
                b->launch.blocks_per_sm = bps_list[pi];
                float ms = 0.0f;
                if ((rc = time_steps(&ms))) break;
                const pbf_batch_tuning r{blocks[bi], order, bps_list[pi], ms, 4};
                if (results && count < max_results) results[count] = r;
                ++count;
                if (r.ms_per_step < pick.ms_per_step) pick = r;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->launch.block = pick.block;
    b->morton = pick.order;
    b->launch.blocks_per_sm = pick.blocks_per_sm;
    b->neighbour_mode = mode_was;
    b->tuned_mode = mode_was == -1 ? pick.neighbour_mode : 0;
    b->use_graph = graph_was;
    b->invalidate_graph();
    BCK(cudaMemcpyAsync(b->pos, b->save_pos, sizeof(float4) * c, cudaMemcpyDeviceToDevice, b->stream));
    BCK(cudaMemcpyAsync(b->vel, b->save_vel, sizeof(float4) * c, cudaMemcpyDeviceToDevice, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    if (rc) return rc;
    if (num_results) *num_results = std::min(count, max_results);
    if (best) *best = pick;
    return PBF_OK;
}
