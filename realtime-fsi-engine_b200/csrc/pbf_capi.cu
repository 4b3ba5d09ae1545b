// pbf_capi.cu — the engine behind the C ABI of include/pbf_b200.h.
//
// Owns the device buffers of one scene, derives the solver constants exactly
// as PBFluids::setParams does (src/fluid/PBFluids.cpp:39-109), and issues the
// substep pipeline of PBFluids::step (src/fluid/PBFluids.cpp:323-517) on one
// CUDA stream:
//
//   for each substep:
//     predict+hash -> radix sort (ceil(log2 H) bits) -> cell table
//     -> reorder into sorted float4 SoA
//     -> I x (lambda, deltaP+apply)  [Jacobi ping-pong]
//     -> integrate (commits x, v to particle order)
//   vorticity confinement (once per step)
//
// The whole step can be replayed from a CUDA graph (pbf_set_use_graph).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pbf_b200.h"
#include "pbf_engine.h"
#include "pbf_kernels.h"

using namespace pbf;

static thread_local std::string g_last_error;

int pbf::set_error(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

#define CHECK_HANDLE(h)                                                                            \
    do {                                                                                           \
        if (!(h)) return pbf::set_error(PBF_ERR_INVALID, "null handle");                           \
        cudaError_t e_ = cudaSetDevice((h)->device);                                               \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_));      \
    } while (0)

// ---- parameter derivation (PBFluids::setParams / setBounds) ------------------

extern "C" int pbf_default_config(pbf_fluid_config* o)
{
    if (!o) return set_error(PBF_ERR_INVALID, "null config");
    std::memset(o, 0, sizeof(*o));
    // include/core/config.h:11-62
    o->dt = 1.0f / 60.0f;
    o->gravity[0] = 0.0f; o->gravity[1] = -3.81f; o->gravity[2] = 0.0f;
    o->h = 0.15f;
    o->rho0 = 1200.0f;
    o->solver_iterations = 3;
    o->substep_iterations = 2;
    o->eps = 0.0001f;
    o->particle_count = 1u << 12;
    o->spawn_min[0] = 2.f; o->spawn_min[1] = 0.2f; o->spawn_min[2] = 2.f;
    o->spawn_max[0] = 5.f; o->spawn_max[1] = 5.f; o->spawn_max[2] = 5.f;
    o->spawn_random = 0;
    o->spacing = 0.1f;
    o->bounds_max[0] = o->bounds_max[1] = o->bounds_max[2] = 6.0f;
    o->bound_damping = 0.5f;
    o->hash_size = 1u << 17;
    o->enable_scorr = 1;
    o->k_corr = 0.001f;
    o->n_corr = 4.0f;
    o->delta_q = 0.3f;
    o->cohesion_strength = 0.001f;
    o->enable_viscosity = 1;
    o->viscosity = 0.1f;
    o->interaction_radius = 1.5f;
    o->interaction_strength = 25.0f;
    o->enable_vorticity = 1;
    o->vorticity_epsilon = 0.05f;
    o->enable_apbf = 0;
    o->min_lod = 2;
    o->max_lod = 7;
    o->lod_max_dist = 15.0f;
    return PBF_OK;
}

static int validate_config(const pbf_fluid_config* c)
{
    if (!c) return set_error(PBF_ERR_INVALID, "null config");
    if (c->hash_size == 0 || (c->hash_size & (c->hash_size - 1u)) != 0)
        return set_error(PBF_ERR_INVALID, "hash_size %u is not a power of two", c->hash_size);
    if (c->hash_size > (1u << 30)) return set_error(PBF_ERR_INVALID, "hash_size %u too large", c->hash_size);
    if (c->substep_iterations == 0) return set_error(PBF_ERR_INVALID, "substep_iterations must be >= 1");
    if (!(c->h > 0.0f)) return set_error(PBF_ERR_INVALID, "h must be > 0");
    if (!(c->rho0 > 0.0f)) return set_error(PBF_ERR_INVALID, "rho0 must be > 0");
    if (c->enable_apbf && (c->max_lod == 0 || c->min_lod > c->max_lod || !(c->lod_max_dist > 0.0f)))
        return set_error(PBF_ERR_INVALID, "invalid APBF levels");
    return PBF_OK;
}

extern "C" int pbf_derive_params(const pbf_fluid_config* c, float pad, pbf_derived_params* u)
{
    if (!c || !u) return set_error(PBF_ERR_INVALID, "null argument");
    std::memset(u, 0, sizeof(*u));
    // setBounds (PBFluids.cpp:299-306)
    for (int a = 0; a < 3; ++a) {
        u->bounds_min[a] = c->bounds_min[a] + pad;
        u->bounds_max[a] = c->bounds_max[a] - pad;
        u->gravity_dt[a] = c->gravity[a];
    }
    const float damping = std::min(std::max(c->bound_damping, 0.0f), 1.0f);
    u->gravity_dt[3] = c->substep_iterations ? c->dt / (float)c->substep_iterations : 0.0f;  // :52
    // wq = calcSCorrKernel(make_pvec3(dq, 0, 0), h)  (PBFluids.cpp:45-46 -> Kernels.cpp:9-27)
    {
        const float pi = 3.14159265358979323846f;
        const float coeff = 315.0f / (64.0f * pi);
        const float h = c->h;
        const float dq = c->delta_q * h;
        const float h2 = h * h;
        const float r2 = dq * dq + 0.0f * 0.0f + 0.0f * 0.0f;
        if (r2 > h2) {
            u->wq = 0.0f;
        } else {
            const float h4 = h2 * h2;
            const float h9 = h4 * h4 * h;
            const float diff = h2 - r2;
            const float diff3 = diff * diff * diff;
            u->wq = (coeff / h9) * diff3;
        }
    }
    u->h = c->h;
    u->rho0 = c->rho0;
    u->eps = c->eps;
    u->k_corr = c->k_corr;
    u->n_corr = c->n_corr;
    u->viscosity = c->viscosity;
    u->bound_damping = damping;
    u->hash_size = c->hash_size;
    u->particle_count = c->particle_count;
    u->enable_scorr = c->enable_scorr ? 1u : 0u;
    u->enable_viscosity = c->enable_viscosity ? 1u : 0u;
    u->cohesion_strength = c->cohesion_strength;
    u->interaction_radius = c->interaction_radius;
    u->interaction_strength = c->interaction_strength;
    // PBFluids.cpp:74-92
    const float PI = 3.14159265358979323846f;
    const float h = c->h;
    const float h2 = h * h;
    const float h3 = h2 * h;
    const float h6 = h3 * h3;
    const float h9 = h6 * h3;
    u->w0_self = (315.0f / (64.0f * PI)) / h3;
    u->poly6_coeff = 315.0f / (64.0f * PI * h9);
    u->spiky_coeff = 45.0f / (PI * h6);
    u->inv_rho0 = 1.0f / c->rho0;
    u->hash_mask = c->hash_size - 1u;
    u->min_lod = c->enable_apbf ? c->min_lod : c->solver_iterations;
    u->max_lod = c->enable_apbf ? c->max_lod : c->solver_iterations;
    u->lod_max_dist = c->lod_max_dist;
    u->enable_apbf = c->enable_apbf ? 1u : 0u;
    return PBF_OK;
}

// ---- handle --------------------------------------------------------------------

template <class T>
static int dalloc(T*& p, size_t count)
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
static void dfree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

DevParams pbf_handle::dev_params() const
{
    DevParams P;
    std::memset(&P, 0, sizeof(P));
    for (int a = 0; a < 3; ++a) {
        P.bmin[a] = derived.bounds_min[a];
        P.bmax[a] = derived.bounds_max[a];
        P.g[a] = derived.gravity_dt[a];
        P.ipos[a] = interaction_pos[a];
        P.cam[a] = camera[a];
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
    P.interacting = interacting ? 1u : 0u;
    P.i_radius = derived.interaction_radius;
    P.i_strength = derived.interaction_strength;
    P.lod_max_dist = derived.lod_max_dist;
    P.min_lod = derived.min_lod;
    P.max_lod = derived.max_lod;
    P.sdf = sdf_dev();
    P.dpb = dpb;
    return P;
}

SdfDev pbf_handle::sdf_dev() const
{
    SdfDev S;
    std::memset(&S, 0, sizeof(S));
    const pbf_handle* o = sdf_src;
    if (!o || !o->grid || !o->sdf_attached) return S;
    S.dist = o->grid;
    S.slab_min = o->slab_min;
    S.dx = o->dims[0];
    S.dy = o->dims[1];
    S.dz = o->dims[2];
    S.ox = o->origin[0];
    S.oy = o->origin[1];
    S.oz = o->origin[2];
    S.cell = o->cell;
    S.inv_cell = 1.0f / o->cell;
    S.padding = sdf_padding;
    S.containment = sdf_containment ? 1 : 0;
    S.enabled = 1;
    return S;
}

int pbf_handle::ensure_capacity(uint32_t need_n)
{
    int rc = PBF_OK;
    if (need_n > cap_n) {
        const size_t c = need_n;
        if ((rc = dalloc(pos, c)) || (rc = dalloc(vel, c)) || (rc = dalloc(pred, c)) || (rc = dalloc(aos, 3 * c)) ||
            (rc = dalloc(keys, c)) || (rc = dalloc(ka, c)) || (rc = dalloc(mcode, c)) || (rc = dalloc(mka, c)) ||
            (rc = dalloc(mia, c)) || (rc = dalloc(mkb, c)) || (rc = dalloc(mib, c)) || (rc = dalloc(ia, c)) || (rc = dalloc(kb, c)) || (rc = dalloc(ib, c)) || (rc = dalloc(sx[0], c)) ||
            (rc = dalloc(sx[1], c)) || (rc = dalloc(sv, c)) || (rc = dalloc(sx0, c)) || (rc = dalloc(somega, c)) || (rc = dalloc(dpb, c)) ||
            (rc = dalloc(rho, c)) || (rc = dalloc(lod, c)) || (rc = dalloc(cand, 2 * c)) ||
            (rc = dalloc(ct_counts, (size_t)contact_num_blocks(need_n) + 1)))
            return rc;
        if ((rc = dalloc(hist, (size_t)256 * sort_num_tiles(need_n)))) return rc;
        cap_n = need_n;
    }
    if (!totals && (rc = dalloc(totals, 256))) return rc;
    if (!scalars && (rc = dalloc(scalars, 8))) return rc;
    if (derived.hash_size != cap_h) {
        if ((rc = dalloc(table, derived.hash_size))) return rc;
        cap_h = derived.hash_size;
    }
    return PBF_OK;
}

void pbf_handle::invalidate_graph()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
}

pbf_handle::~pbf_handle()
{
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    invalidate_graph();
    for (auto& r : prof_pending) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    dfree(pos); dfree(vel); dfree(pred); dfree(aos); dfree(keys);
    dfree(mcode); dfree(mka); dfree(mia); dfree(mkb); dfree(mib); dfree(ka); dfree(ia); dfree(kb); dfree(ib);
    dfree(sx[0]); dfree(sx[1]); dfree(sv); dfree(sx0); dfree(somega); dfree(dpb); dfree(rho); dfree(lod);
    dfree(hist); dfree(totals); dfree(table); dfree(cand); dfree(ct_counts); dfree(scalars);
    dfree(lx[0]); dfree(lx[1]); dfree(lxb); dfree(lv); dfree(lx0); dfree(lom); dfree(lrho);
    dfree(lid); dfree(lkey); dfree(inv); dfree(dkey_id);
    dfree(dtable); dfree(druns); dfree(dclean); dfree(ddcol); dfree(ddirty); dfree(dflag);
    dfree(dslot); dfree(dord); dfree(dcnt); dfree(dbsum); dfree(dhm); dfree(dhcnt); dfree(dvmark);
    dfree(grid); dfree(slab_min);
    mesh_free();
    if (stream) cudaStreamDestroy(stream);
}

// ---- profiling ----------------------------------------------------------------------
cudaEvent_t pbf_handle::take_event()
{
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void pbf_handle::prof_begin(int slot)
{
    if (!profiling || capturing) return;
    ProfRec r;
    r.slot = slot;
    r.a = take_event();
    r.b = nullptr;
    cudaEventRecord(r.a, stream);
    prof_open[slot] = (int)prof_pending.size();
    prof_pending.push_back(r);
}

void pbf_handle::prof_end(int slot)
{
    if (!profiling || capturing) return;
    const int i = prof_open[slot];
    if (i < 0 || i >= (int)prof_pending.size()) return;
    prof_pending[i].b = take_event();
    cudaEventRecord(prof_pending[i].b, stream);
    prof_open[slot] = -1;
}

int pbf_handle::prof_collect()
{
    CK(cudaStreamSynchronize(stream));
    for (auto& r : prof_pending) {
        if (r.b) {
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, r.a, r.b));
            prof_ms[r.slot] += ms;
            prof_count[r.slot] += 1;
            event_pool.push_back(r.b);
        }
        event_pool.push_back(r.a);
    }
    prof_pending.clear();
    return PBF_OK;
}

// ---- neighbour-pass mode -----------------------------------------------------------------
// Mode 8 (dense-window runs) needs label arrays without APBF's per-particle
// skips and a dense window of the box within 2^26 cells; otherwise the
// handle runs mode 4 (hashed buckets).  Automatic choice (the default,
// pass_mode < 0): mode 8 from 2^19 particles, below which its extra
// relabelling launches cost more than its walk saves (measured crossover
// between 2.6e5 and 8.8e5 particles), mode 4 below.
int pbf_handle::effective_mode() const
{
    const int mode = pass_mode >= 0 ? pass_mode : (n >= (1u << 19) ? 8 : 4);
    if (mode == 8 && (derived.enable_apbf || n >= (1u << 27))) return 4;
    if (mode == 8) {
        int g0[3];
        uint32_t nd[3];
        if (!dense_window(g0, nd)) return 4;
    }
    return mode;
}

int pbf_handle::ensure_label_capacity()
{
    int rc;
    if (cap_label_n < n || !inv) {
        // (kLabelPad entries past the last label: a run's last chunk loads them and masks them out)
        const size_t c = std::max<uint32_t>(n, 1u), cp = c + kLabelPad;
        if ((rc = dalloc(lx[0], cp)) || (rc = dalloc(lx[1], cp)) || (rc = dalloc(lxb, c)) || (rc = dalloc(lv, cp)) ||
            (rc = dalloc(lx0, cp)) || (rc = dalloc(lom, cp)) || (rc = dalloc(lrho, c)) || (rc = dalloc(lid, c)) ||
            (rc = dalloc(lkey, c)) || (rc = dalloc(inv, c)) || (rc = dalloc(dkey_id, c)))
            return rc;
        dkey_valid = false;
        cap_label_n = (uint32_t)c;
    }
    return PBF_OK;
}

// ---- dense cell window (mode 8) -----------------------------------------------------------
// The walls' box in cells (floor(x / h) in FP32, as the kernels compute a
// cell) with kDenseMargin cells of margin on each side.  Any window is
// correct (cells outside wrap into it and their queries walk the hashed
// buckets); the margin also holds the predict-time cells of particles that
// move towards a wall (x* = x + v dt lies beyond it until the walls clamp
// it), whose later correction would otherwise count as an unchecked drift.

bool pbf_handle::dense_window(int g0[3], uint32_t nd[3]) const
{
    const float h = derived.h;
    if (!(h > 0.0f)) return false;
    uint64_t slots = 1;
    for (int a = 0; a < 3; ++a) {
        const float lo = std::floor(derived.bounds_min[a] / h), hi = std::floor(derived.bounds_max[a] / h);
        if (!(lo >= -1e8f && hi <= 1e8f && hi >= lo)) return false;
        g0[a] = (int)lo - kDenseMargin;
        nd[a] = (uint32_t)((int)hi - (int)lo + 1 + 2 * kDenseMargin);
        slots *= nd[a];
    }
    return slots <= (1ull << 26);
}

DenseArgs pbf_handle::dense_args() const
{
    DenseArgs D;
    D.table = dtable;
    D.runs = druns;
    D.order = nullptr;
    D.hm = dhm;
    D.hcnt = dhcnt;
    D.use_list = 0;
    D.rec_slot = nullptr;
    D.rec_cnt = nullptr;
    D.clean = dclean;
    D.dcol = ddcol;
    D.dirty = ddirty;
    D.rec_list = 0;
    D.vmark = dvmark;
    D.htable = table;
    D.inv = inv;
    D.xb = lxb;
    D.flag = dflag;
    D.gx0 = dwin_g0[0];
    D.gy0 = dwin_g0[1];
    D.gz0 = dwin_g0[2];
    D.nx = dwin_n[0];
    D.ny = dwin_n[1];
    D.nz = dwin_n[2];
    const float b = 0.9f * derived.h;
    D.drift2 = b * b;
    D.slot0 = 0;
    D.total = dwin_n[0] * dwin_n[1] * dwin_n[2];
    D.scenes = nullptr;
    D.scene_of = nullptr;
    D.slot_scene = nullptr;
    return D;
}

// Buffers of mode 8 and the per-slot flags of the current window and hash
// mask; recomputed (one kernel, then a synchronize) when either changes.  Runs
// before any graph capture of the step.
int pbf_handle::ensure_dense()
{
    int rc;
    if ((rc = ensure_label_capacity())) return rc;
    if (cap_ord_n < n || !dord) {
        if (capturing) return set_error(PBF_ERR_INVALID, "particle count grew during graph capture");
        const size_t c = std::max<uint32_t>(n, 1u);
        if ((rc = dalloc(dslot, c)) || (rc = dalloc(dord, c)) || (rc = dalloc(dhm, c * kDenseListWords)) ||
            (rc = dalloc(dhcnt, c)))
            return rc;
        cap_ord_n = (uint32_t)c;
    }
    int g0[3];
    uint32_t nd[3];
    if (!dense_window(g0, nd)) return set_error(PBF_ERR_INVALID, "dense cell window larger than 2^26 cells");
    const size_t slots = (size_t)nd[0] * nd[1] * nd[2];
    const bool same = dwin_ready && dwin_mask == derived.hash_size - 1 && std::equal(g0, g0 + 3, dwin_g0) &&
                      std::equal(nd, nd + 3, dwin_n);
    if (same) return PBF_OK;
    if (capturing) return set_error(PBF_ERR_INVALID, "dense cell window changed during graph capture");
    if (slots > cap_slots || !dtable) {
        if ((rc = dalloc(dtable, slots + 1)) || (rc = dalloc(druns, slots)) || (rc = dalloc(dcnt, slots + 1)) ||
            (rc = dalloc(dbsum, order_scan_blocks((uint32_t)slots))) || (rc = dalloc(dclean, slots)) ||
            (rc = dalloc(ddcol, slots)) ||
            (rc = dalloc(ddirty, slots)) || (rc = dalloc(dvmark, slots)))
            return rc;
        cap_slots = slots;
    }
    if (!dflag && (rc = dalloc(dflag, 4))) return rc;
    std::copy(g0, g0 + 3, dwin_g0);
    std::copy(nd, nd + 3, dwin_n);
    dwin_mask = derived.hash_size - 1;
    CK(cudaMemsetAsync(dflag, 0, 4 * sizeof(uint32_t), stream));
    launch_d_clean(dense_args(), dwin_mask, dclean, dflag + 2, num_sms, stream);
    launch_d_dcol(dense_args(), dwin_mask, ddcol, num_sms, stream);
    launches += 2;
    CK(cudaMemcpyAsync(&dwin_unclean, dflag + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    dwin_ready = true;
    return PBF_OK;
}

// Sorted-order buffers are kept in label order in mode 8: gather the one asked
// for back into sorted (hash) order before it is read.
int pbf_handle::unpermute_for_read(int which)
{
    if (!label_space) return PBF_OK;
    switch (which) {
    case PBF_BUF_XSTAR:
        launch_d_unpermute4(n, inv, lx[last_x], sx[last_x], num_sms, stream);
        break;
    case PBF_BUF_RHO:
        launch_d_unpermute1(n, inv, lrho, rho, num_sms, stream);
        break;
    case PBF_BUF_OMEGA:
        launch_d_unpermute4(n, inv, lom, somega, num_sms, stream);
        break;
    case PBF_BUF_VPRED:
        launch_d_unpermute4(n, inv, lv, sv, num_sms, stream);
        break;
    default:
        return PBF_OK;
    }
    ++launches;
    CK(cudaStreamSynchronize(stream));
    return PBF_OK;
}

// ---- pipeline -------------------------------------------------------------------------
int pbf_handle::stage(int st, uint32_t iter)
{
    const DevParams P = dev_params();
    const int sms = num_sms;
    const int mode = effective_mode();
    if (mode == 8 && st >= PBF_STAGE_LAMBDA && st <= PBF_STAGE_VORTICITY) {
        if (!label_space || !dwin_ready) return set_error(PBF_ERR_INVALID, "mode 8: run the reorder stage first");
        DenseArgs D = dense_args();
        prof_begin(st);
        // after the first iteration the particles have moved off their
        // predict-time cells: threads take them by current cell (lambda
        // computes the order, the delta-p of the same iteration reuses it)
        // (a pass that moves particles records the slots of its outputs, so the
        // order of the next pass needs only the scan and the placement)
        auto order_by = [&](const float4* X) {
            if (dslot_fresh)
                launch_d_order_recorded(P, D, dslot, dcnt, dbsum, dord, stream, &launches);
            else
                launch_d_order(P, D, X, dslot, dcnt, dbsum, dord, stream, &launches);
            dslot_fresh = false;
            D.order = dord;
        };
        const size_t slots = (size_t)dwin_n[0] * dwin_n[1] * dwin_n[2];
        auto record_next = [&]() -> int {
            CK(cudaMemsetAsync(dcnt, 0, sizeof(uint32_t) * (slots + 1), stream));
            D.rec_slot = dslot;
            D.rec_cnt = dcnt;
            dslot_fresh = true;
            return PBF_OK;
        };
        switch (st) {
        case PBF_STAGE_LAMBDA:
            if (iter >= 2) {
                order_by(lx[0]);
                dord_iter = (int)iter;
            }
            launch_d_lambda(P, D, lx[0], lx[1], lrho, stream);
            dlist_iter = (int)iter;
            last_x = 1;
            break;
        case PBF_STAGE_DELTAP:
            if (iter >= 2 && dord_iter == (int)iter) D.order = dord;
            D.use_list = dlist_iter == (int)iter ? 1 : 0;
            dlist_iter = 0;
            if (const int rc = record_next()) return rc;
            launch_d_deltap(P, D, lx[1], lx[0], stream);
            last_x = 0;
            break;
        case PBF_STAGE_INTEGRATE:
            order_by(lx[0]);
            dord_iter = 0;
            dlist_iter = 0;
            if (P.vort_on) {
                if (const int rc = record_next()) return rc;
                // hit masks for the vorticity pass
                CK(cudaMemsetAsync(dvmark, 0, slots, stream));
                D.rec_list = 1;
                dvlist_ready = true;
            }
            launch_d_integrate(P, D, lx[0], lv, lx0, lom, lid, pos, vel, stream);
            break;
        default:
            order_by(lx0);
            dord_iter = 0;
            D.use_list = dvlist_ready ? 1 : 0;
            dvlist_ready = false;
            launch_d_vorticity(P, D, lx0, lom, lid, vel, stream);
            break;
        }
        ++launches;
        prof_end(st);
        return PBF_OK;
    }
    switch (st) {
    case PBF_STAGE_PREDICT:
        prof_begin(PBF_STAGE_PREDICT);
        dkey_valid = false;
        if (mode == 8 && dwin_ready && dkey_id && cap_label_n >= n) {
            launch_d_predict_hash(P, dense_args(), pos, vel, keys, dkey_id, sms, stream);
            dkey_valid = true;
            dkey_gen = particles_gen;
            dkey_P = P;
            std::copy(dwin_g0, dwin_g0 + 3, dkey_g0);
            std::copy(dwin_n, dwin_n + 3, dkey_n);
        } else {
            launch_predict_hash(P, pos, vel, keys, sms, stream);
        }
        ++launches;
        prof_end(PBF_STAGE_PREDICT);
        break;
    case PBF_STAGE_SORT: {
        prof_begin(PBF_STAGE_SORT);
        uint32_t bits = 0;
        while ((1u << bits) < derived.hash_size) ++bits;
        launch_radix_sort(n, bits, keys, ka, ia, kb, ib, hist, totals, &skeys, &ids, stream, &launches);
        prof_end(PBF_STAGE_SORT);
        break;
    }
    case PBF_STAGE_TABLE:
        prof_begin(PBF_STAGE_TABLE);
        CK(cudaMemsetAsync(table, 0xFF, sizeof(int2) * (size_t)derived.hash_size, stream));
        launch_build_table(n, skeys, table, sms, stream);
        ++launches;
        prof_end(PBF_STAGE_TABLE);
        break;
    case PBF_STAGE_REORDER:
        prof_begin(PBF_STAGE_REORDER);
        order = nullptr;
        if (mode == 8) {
            // relabel by window slot, then the slot table of the labels (the
            // hash-sorted arrays are not needed: keys and label-order arrays
            // come straight from the particle state)
            int rc = ensure_dense();
            if (rc) return rc;
            const DenseArgs D = dense_args();
            // the predict pass's slots when nothing they depend on changed since
            const bool reuse = dkey_valid && dkey_gen == particles_gen &&
                               std::memcmp(&dkey_P, &P, sizeof(DevParams)) == 0 &&
                               std::equal(dkey_g0, dkey_g0 + 3, dwin_g0) && std::equal(dkey_n, dkey_n + 3, dwin_n);
            dkey_valid = false;
            if (reuse)
                launch_d_keys_gather(n, ids, dkey_id, mcode, sms, stream);
            else
                launch_d_keys_pred(P, D, ids, pos, vel, mcode, sms, stream);
            ++launches;
            const uint64_t slots = (uint64_t)dwin_n[0] * dwin_n[1] * dwin_n[2];
            uint32_t* msorted = mka;
            if ((uint64_t)derived.hash_size * 64u >= n) {
                // labels by counting (launch_d_relabel), into the relabelling's sort
                // buffers; each particle scans the part of its bucket before it, so
                // the buckets must stay short
                order = mia;
                launch_d_relabel(n, (uint32_t)slots, mcode, skeys, dcnt, dbsum, dflag + 3, order, msorted, sms,
                                 stream, &launches);
            } else {
                // a hash table far smaller than the particle count: a stable radix
                // sort of the keys (the overflow key `slots` included)
                uint32_t bits = 1;
                while ((1ull << bits) <= slots) ++bits;
                launch_radix_sort(n, bits, mcode, mka, mia, mkb, mib, hist, totals, &msorted, &order, stream,
                                  &launches);
            }
            launch_d_permute(P, order, ids, skeys, pos, vel, lx[0], lxb, lv, lx0, lid, lkey, inv, sms, stream);
            ++launches;
            // (slot `slots` holds the overflow's labels)
            CK(cudaMemsetAsync(dtable, 0xFF, sizeof(int2) * (slots + 1), stream));
            launch_build_table(n, msorted, dtable, sms, stream);
            launch_d_runs(dense_args(), dtable, druns, sms, stream);
            launches += 2;
            CK(cudaMemsetAsync(ddirty, 0, sizeof(uint32_t) * slots, stream));
            dord_iter = 0;
            dlist_iter = 0;
            dvlist_ready = false;
            dslot_fresh = false;
            CK(cudaMemsetAsync(dflag, 0, sizeof(uint32_t), stream));
            label_space = true;
            last_x = 0;
            prof_end(PBF_STAGE_REORDER);
            break;
        }
        launch_reorder(P, ids, pos, vel, sx[0], sv, sx0, lod, mcode, sms, stream);
        ++launches;
        {
            uint32_t* msorted = nullptr;
            launch_radix_sort(n, 24, mcode, mka, mia, mkb, mib, hist, totals, &msorted, &order, stream, &launches);
        }
        label_space = false;
        last_x = 0;
        prof_end(PBF_STAGE_REORDER);
        break;
    case PBF_STAGE_LAMBDA:
        prof_begin(PBF_STAGE_LAMBDA);
        launch_lambda_m(P, sx[0], sx[1], rho, table, lod, iter, order, stream);
        ++launches;
        last_x = 1;
        prof_end(PBF_STAGE_LAMBDA);
        break;
    case PBF_STAGE_DELTAP:
        prof_begin(PBF_STAGE_DELTAP);
        launch_deltap_m(P, sx[1], sx[0], table, lod, iter, order, stream);
        ++launches;
        last_x = 0;
        prof_end(PBF_STAGE_DELTAP);
        break;
    case PBF_STAGE_INTEGRATE:
        prof_begin(PBF_STAGE_INTEGRATE);
        launch_integrate_m(P, sx[0], sv, sx0, somega, ids, pos, vel, table, order, stream);
        ++launches;
        prof_end(PBF_STAGE_INTEGRATE);
        break;
    case PBF_STAGE_VORTICITY:
        prof_begin(PBF_STAGE_VORTICITY);
        launch_vorticity_m(P, sx0, somega, ids, vel, table, order, stream);
        ++launches;
        prof_end(PBF_STAGE_VORTICITY);
        break;
    default:
        return set_error(PBF_ERR_INVALID, "unknown stage %d", st);
    }
    return PBF_OK;
}

int pbf_handle::step_body()
{
    int rc;
    const uint32_t max_iter = derived.enable_apbf ? derived.max_lod : cfg.solver_iterations;  // :455
    for (uint32_t s = 0; s < cfg.substep_iterations; ++s) {
        if ((rc = stage(PBF_STAGE_PREDICT, 0)) || (rc = stage(PBF_STAGE_SORT, 0)) || (rc = stage(PBF_STAGE_TABLE, 0)) ||
            (rc = stage(PBF_STAGE_REORDER, 0)))
            return rc;
        for (uint32_t it = 1; it <= max_iter; ++it)
            if ((rc = stage(PBF_STAGE_LAMBDA, it)) || (rc = stage(PBF_STAGE_DELTAP, it))) return rc;
        if ((rc = stage(PBF_STAGE_INTEGRATE, 0))) return rc;
    }
    if (cfg.enable_vorticity && (rc = stage(PBF_STAGE_VORTICITY, 0))) return rc;
    return PBF_OK;
}

int pbf_handle::step()
{
    if (n == 0) return PBF_OK;  // PBFluids.cpp:325
    if (effective_mode() == 8) {
        const int rc = ensure_dense();  // allocation and slot flags before any capture
        if (rc) return rc;
    }
    const uint64_t gen = sdf_src ? sdf_src->grid_generation : 0;
    if (graph_exec && gen != captured_generation) invalidate_graph();
    if (use_graph) {
        captured_generation = gen;
        if (!graph_exec) {
            const uint64_t before = launches;
            capturing = true;
            CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
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
            CK(cudaGraphInstantiate(&graph_exec, graph, 0));
            graph_launches = launches - before;
            launches = before;
        }
        prof_begin(0);
        CK(cudaGraphLaunch(graph_exec, stream));
        prof_end(0);
        launches += graph_launches;
    } else {
        prof_begin(0);
        const int rc = step_body();
        prof_end(0);
        if (rc) return rc;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return PBF_OK;
}

// ---- C ABI -----------------------------------------------------------------------------
extern "C" int pbf_abi_version(void) { return PBF_ABI_VERSION; }
extern "C" const char* pbf_last_error(void) { return g_last_error.c_str(); }

extern "C" int pbf_create(const pbf_fluid_config* cfg, int device, pbf_handle** out)
{
    if (!out) return set_error(PBF_ERR_INVALID, "null output handle");
    *out = nullptr;
    int rc = validate_config(cfg);
    if (rc) return rc;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return set_error(PBF_ERR_INVALID, "device %d out of range (%d)", device, ndev);
    CK(cudaSetDevice(device));
    pbf_handle* h = new pbf_handle();
    h->device = device;
    h->cfg = *cfg;
    for (int i = 0; i < PBF_NUM_PASS_SLOTS; ++i) h->prof_open[i] = -1;
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return set_error(PBF_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
    }
    pbf_derive_params(&h->cfg, h->collision_padding, &h->derived);
    *out = h;
    return PBF_OK;
}

extern "C" int pbf_destroy(pbf_handle* h)
{
    if (!h) return PBF_OK;
    delete h;
    return PBF_OK;
}

extern "C" int pbf_set_params(pbf_handle* h, const pbf_fluid_config* cfg)
{
    CHECK_HANDLE(h);
    int rc = validate_config(cfg);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    h->cfg = *cfg;
    h->cfg.particle_count = h->n ? h->n : cfg->particle_count;
    pbf_derive_params(&h->cfg, h->collision_padding, &h->derived);
    h->invalidate_graph();
    if (h->n && (rc = h->ensure_capacity(h->n))) return rc;
    return PBF_OK;
}

extern "C" int pbf_get_params(pbf_handle* h, pbf_fluid_config* out)
{
    if (!h || !out) return set_error(PBF_ERR_INVALID, "null argument");
    *out = h->cfg;
    return PBF_OK;
}

extern "C" int pbf_get_derived(pbf_handle* h, pbf_derived_params* out)
{
    if (!h || !out) return set_error(PBF_ERR_INVALID, "null argument");
    *out = h->derived;
    return PBF_OK;
}

// setBounds applies immediately (the reference stores the values and uploads
// them with the next setParams; its only caller passes the FluidConfig bounds).
extern "C" int pbf_set_bounds(pbf_handle* h, const float mn[3], const float mx[3], float damping)
{
    if (!h || !mn || !mx) return set_error(PBF_ERR_INVALID, "null argument");
    for (int a = 0; a < 3; ++a) {
        h->derived.bounds_min[a] = mn[a] + h->collision_padding;
        h->derived.bounds_max[a] = mx[a] - h->collision_padding;
    }
    h->derived.bound_damping = std::min(std::max(damping, 0.0f), 1.0f);
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_set_collision_padding(pbf_handle* h, float p)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    h->collision_padding = p;  // takes effect at the next setParams / setBounds (PBFluids.h:108-112)
    return PBF_OK;
}

extern "C" int pbf_set_camera_pos(pbf_handle* h, const float p[3])
{
    if (!h || !p) return set_error(PBF_ERR_INVALID, "null argument");
    for (int a = 0; a < 3; ++a) h->camera[a] = p[a];
    if (h->derived.enable_apbf) h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_set_interaction(pbf_handle* h, int active, const float p[3])
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    h->interacting = active != 0;
    if (p)
        for (int a = 0; a < 3; ++a) h->interaction_pos[a] = p[a];
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_set_particles(pbf_handle* h, const pbf_particle* ps, uint32_t n)
{
    CHECK_HANDLE(h);
    ++h->particles_gen;
    if (n && !ps) return set_error(PBF_ERR_INVALID, "null particles with n=%u", n);
    CK(cudaStreamSynchronize(h->stream));
    h->invalidate_graph();
    h->n = n;
    h->label_space = false;
    h->cfg.particle_count = n;  // PBFluids.cpp:117-118
    pbf_derive_params(&h->cfg, h->collision_padding, &h->derived);
    h->contact_count_host = 0;
    h->contacts_valid = false;
    if (n == 0) return PBF_OK;
    int rc = h->ensure_capacity(n);
    if (rc) return rc;
    // one copy of the Particle array, split into the engine's arrays on the GPU
    CK(cudaMemcpyAsync(h->aos, ps, sizeof(pbf_particle) * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    launch_unpack_particles(n, h->aos, h->pos, h->pred, h->vel, h->num_sms, h->stream);
    ++h->launches;
    CK(cudaMemsetAsync(h->somega, 0, sizeof(float4) * n, h->stream));
    // a delta-p stage run without the lambda stage before it reads zeros, not stale memory
    CK(cudaMemsetAsync(h->dpb, 0, sizeof(float4) * n, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PBF_OK;
}

// Same-size refresh of the particle state from host memory without the
// re-derivation and reallocation of setParticles; used per step by callers
// that own the state on the host.
extern "C" int pbf_upload_particles(pbf_handle* h, const pbf_particle* ps, uint32_t n)
{
    CHECK_HANDLE(h);
    ++h->particles_gen;
    if (n != h->n) return pbf_set_particles(h, ps, n);
    if (n == 0) return PBF_OK;
    if (!ps) return set_error(PBF_ERR_INVALID, "null particles");
    CK(cudaMemcpyAsync(h->aos, ps, sizeof(pbf_particle) * (size_t)n, cudaMemcpyHostToDevice, h->stream));
    launch_unpack_particles(n, h->aos, h->pos, h->pred, h->vel, h->num_sms, h->stream);
    ++h->launches;
    return PBF_OK;
}

extern "C" int pbf_particle_count(pbf_handle* h, uint32_t* n)
{
    if (!h || !n) return set_error(PBF_ERR_INVALID, "null argument");
    *n = h->n;
    return PBF_OK;
}

extern "C" int pbf_read_particles(pbf_handle* h, pbf_particle* out, uint32_t n)
{
    CHECK_HANDLE(h);
    if (n != h->n) return set_error(PBF_ERR_INVALID, "read_particles: n=%u but the scene holds %u", n, h->n);
    if (n == 0) return PBF_OK;
    if (!out) return set_error(PBF_ERR_INVALID, "null output");
    launch_pack_particles(n, h->pos, h->pred, h->vel, h->aos, h->num_sms, h->stream);
    ++h->launches;
    CK(cudaMemcpyAsync(out, h->aos, sizeof(pbf_particle) * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PBF_OK;
}

extern "C" int pbf_set_particles_device(pbf_handle* h, const void* pos4, const void* vel4, uint32_t n)
{
    CHECK_HANDLE(h);
    ++h->particles_gen;
    if (n && (!pos4 || !vel4)) return set_error(PBF_ERR_INVALID, "null device pointers");
    if (n != h->n) {
        CK(cudaStreamSynchronize(h->stream));
        h->invalidate_graph();
        h->n = n;
        h->label_space = false;
        h->cfg.particle_count = n;
        pbf_derive_params(&h->cfg, h->collision_padding, &h->derived);
        if (n) {
            int rc = h->ensure_capacity(n);
            if (rc) return rc;
            CK(cudaMemsetAsync(h->pred, 0, sizeof(float4) * n, h->stream));
            CK(cudaMemsetAsync(h->dpb, 0, sizeof(float4) * n, h->stream));
        }
    }
    if (n == 0) return PBF_OK;
    CK(cudaMemcpyAsync(h->pos, pos4, sizeof(float4) * n, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->vel, vel4, sizeof(float4) * n, cudaMemcpyDeviceToDevice, h->stream));
    return PBF_OK;
}

extern "C" int pbf_read_particles_device(pbf_handle* h, void* pos4, void* vel4, uint32_t n)
{
    CHECK_HANDLE(h);
    if (n != h->n) return set_error(PBF_ERR_INVALID, "n mismatch");
    if (n == 0) return PBF_OK;
    if (pos4) CK(cudaMemcpyAsync(pos4, h->pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, h->stream));
    if (vel4) CK(cudaMemcpyAsync(vel4, h->vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, h->stream));
    return PBF_OK;
}

extern "C" int pbf_step(pbf_handle* h)
{
    CHECK_HANDLE(h);
    return h->step();
}

extern "C" int pbf_sync(pbf_handle* h)
{
    CHECK_HANDLE(h);
    CK(cudaStreamSynchronize(h->stream));
    return PBF_OK;
}

extern "C" int pbf_get_stream(pbf_handle* h, void** s)
{
    if (!h || !s) return set_error(PBF_ERR_INVALID, "null argument");
    *s = (void*)h->stream;
    return PBF_OK;
}

// ---- SDF grid ------------------------------------------------------------------------
int pbf_handle::upload_grid(const float* dist_host, const int32_t d[3], const float o[3], float c)
{
    const size_t total = (size_t)d[0] * d[1] * d[2];
    int rc;
    if (total != grid_elems) {
        if ((rc = dalloc(grid, total))) return rc;
        grid_elems = total;
        ++grid_generation;
    }
    if (!slab_min && (rc = dalloc(slab_min, 6))) return rc;
    for (int a = 0; a < 3; ++a) {
        dims[a] = d[a];
        origin[a] = o[a];
    }
    cell = c;
    if (dist_host) CK(cudaMemcpyAsync(grid, dist_host, total * sizeof(float), cudaMemcpyHostToDevice, stream));
    launch_sdf_slab_min(grid, dims[0], dims[1], dims[2], slab_min, stream);
    ++launches;
    sdf_attached = true;
    sdf_src = this;
    invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_set_sdf_grid(pbf_handle* h, const float* dist, const int32_t dims[3], const float origin[3],
                                float cell)
{
    CHECK_HANDLE(h);
    if (!dist || !dims || !origin) return set_error(PBF_ERR_INVALID, "null argument");
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) return set_error(PBF_ERR_INVALID, "bad SDF dims");
    if ((size_t)dims[0] * dims[1] * dims[2] > (size_t)1 << 31) return set_error(PBF_ERR_INVALID, "SDF grid too large");
    if (!(cell > 0.0f)) return set_error(PBF_ERR_INVALID, "SDF cell size must be > 0");
    CK(cudaStreamSynchronize(h->stream));
    h->mesh_attached = false;
    int rc = h->upload_grid(dist, dims, origin, cell);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return PBF_OK;
}

extern "C" int pbf_clear_sdf(pbf_handle* h)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    h->sdf_src = nullptr;
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_attach_sdf(pbf_handle* h, pbf_handle* sdf)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    if (sdf && sdf->device != h->device)
        return set_error(PBF_ERR_INVALID, "SDF lives on device %d, fluid on %d", sdf->device, h->device);
    if (sdf && !sdf->grid) return set_error(PBF_ERR_STATE, "SDF handle holds no grid");
    h->sdf_src = sdf;
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_set_sdf_mode(pbf_handle* h, float padding, int containment)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    h->sdf_padding = padding;
    h->sdf_containment = containment != 0;
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_read_sdf_grid(pbf_handle* h, float* out, size_t n)
{
    CHECK_HANDLE(h);
    if (!h->grid) return set_error(PBF_ERR_STATE, "no SDF grid");
    if (n != h->grid_elems || !out) return set_error(PBF_ERR_INVALID, "read_sdf_grid: need %zu floats", h->grid_elems);
    CK(cudaMemcpyAsync(out, h->grid, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PBF_OK;
}

extern "C" int pbf_sample_sdf(pbf_handle* h, const float* pts3, uint32_t n, float* out_d, float* out_g)
{
    CHECK_HANDLE(h);
    if (!h->sdf_dev().enabled) return set_error(PBF_ERR_STATE, "no SDF attached");
    if (n == 0) return PBF_OK;
    if (!pts3 || !out_d) return set_error(PBF_ERR_INVALID, "null argument");
    float *dp = nullptr, *dd = nullptr, *dg = nullptr;
    int rc = PBF_OK;
    if ((rc = dalloc(dp, 3 * (size_t)n)) || (rc = dalloc(dd, n)) || (out_g && (rc = dalloc(dg, 3 * (size_t)n)))) {
        dfree(dp); dfree(dd); dfree(dg);
        return rc;
    }
    cudaMemcpyAsync(dp, pts3, 12 * (size_t)n, cudaMemcpyHostToDevice, h->stream);
    launch_sdf_sample(h->sdf_dev(), dp, n, dd, dg, h->stream);
    ++h->launches;
    cudaMemcpyAsync(out_d, dd, 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream);
    if (out_g) cudaMemcpyAsync(out_g, dg, 12 * (size_t)n, cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    dfree(dp); dfree(dd); dfree(dg);
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "sample_sdf: %s", cudaGetErrorString(e));
    return PBF_OK;
}

// ---- contacts ----------------------------------------------------------------------------
extern "C" int pbf_filter_contacts(pbf_handle* h, float band)
{
    CHECK_HANDLE(h);
    if (!h->sdf_dev().enabled || !(band > 0.0f)) return PBF_OK;  // PBFluids.cpp:195
    if (h->n == 0) return PBF_OK;                                     // PBFluids.cpp:196
    launch_contact_filter(h->sdf_dev(), h->n, h->pos, h->vel, band, h->ct_counts, h->scalars, h->cand, h->stream,
                          &h->launches);
    h->contacts_valid = true;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "contact filter: %s", cudaGetErrorString(e));
    return PBF_OK;
}

extern "C" int pbf_read_contacts(pbf_handle* h, pbf_contact_candidate* out, uint32_t capacity, uint32_t* count)
{
    CHECK_HANDLE(h);
    if (!count) return set_error(PBF_ERR_INVALID, "null count");
    *count = 0;
    if (!h->contacts_valid || h->n == 0) return PBF_OK;
    uint32_t c = 0;
    CK(cudaMemcpyAsync(&c, h->scalars, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    c = std::min(c, h->n);
    *count = c;
    if (out && capacity) {
        const uint32_t m = std::min(c, capacity);
        if (m) {
            CK(cudaMemcpyAsync(out, h->cand, sizeof(pbf_contact_candidate) * m, cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
        }
    }
    return PBF_OK;
}

// ---- stage access ------------------------------------------------------------------------
extern "C" int pbf_run_stage(pbf_handle* h, int stage, uint32_t iter)
{
    CHECK_HANDLE(h);
    if (h->n == 0) return set_error(PBF_ERR_STATE, "no particles");
    if (stage > PBF_STAGE_SORT && !h->ids) return set_error(PBF_ERR_STATE, "stage %d before sort", stage);
    int rc = h->stage(stage, iter);
    if (rc) return rc;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "stage %d: %s", stage, cudaGetErrorString(e));
    return PBF_OK;
}

static int buffer_info(pbf_handle* h, int which, void** p, size_t* bytes)
{
    const size_t n = h->n;
    if (int rc = h->unpermute_for_read(which)) return rc;
    switch (which) {
    case PBF_BUF_KEYS: *p = h->keys; *bytes = 4 * n; break;
    case PBF_BUF_SORTED_KEYS: *p = h->skeys; *bytes = 4 * n; break;
    case PBF_BUF_SORTED_IDS: *p = h->ids; *bytes = 4 * n; break;
    case PBF_BUF_TABLE: *p = h->table; *bytes = 8 * (size_t)h->derived.hash_size; break;
    case PBF_BUF_XSTAR: *p = h->sx[h->last_x]; *bytes = 16 * n; break;
    case PBF_BUF_VPRED: *p = h->sv; *bytes = 16 * n; break;
    case PBF_BUF_RHO: *p = h->rho; *bytes = 4 * n; break;
    case PBF_BUF_OMEGA: *p = h->somega; *bytes = 16 * n; break;
    case PBF_BUF_POS: *p = h->pos; *bytes = 16 * n; break;
    case PBF_BUF_VEL: *p = h->vel; *bytes = 16 * n; break;
    case PBF_BUF_LOD: *p = h->lod; *bytes = 4 * n; break;
    default: return set_error(PBF_ERR_INVALID, "unknown buffer %d", which);
    }
    if (!*p) return set_error(PBF_ERR_STATE, "buffer %d not allocated yet", which);
    return PBF_OK;
}

extern "C" int pbf_read_buffer(pbf_handle* h, int which, void* out, size_t bytes)
{
    CHECK_HANDLE(h);
    void* p = nullptr;
    size_t b = 0;
    int rc = buffer_info(h, which, &p, &b);
    if (rc) return rc;
    if (bytes != b || !out) return set_error(PBF_ERR_INVALID, "buffer %d holds %zu bytes, asked %zu", which, b, bytes);
    CK(cudaMemcpyAsync(out, p, b, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return PBF_OK;
}

extern "C" int pbf_buffer_device_ptr(pbf_handle* h, int which, void** dev, size_t* bytes)
{
    if (!h || !dev || !bytes) return set_error(PBF_ERR_INVALID, "null argument");
    return buffer_info(h, which, dev, bytes);
}

// ---- standalone primitives -------------------------------------------------------------------
extern "C" int pbf_sort_keys(const uint32_t* keys, uint32_t n, uint32_t key_bits, uint32_t* sorted_keys,
                             uint32_t* sorted_ids)
{
    if (n == 0) return PBF_OK;
    if (!keys || !sorted_keys || !sorted_ids) return set_error(PBF_ERR_INVALID, "null argument");
    if (key_bits > 32) return set_error(PBF_ERR_INVALID, "key_bits %u > 32", key_bits);
    if (key_bits < 32)
        for (uint32_t i = 0; i < n; ++i)
            if (keys[i] >> key_bits) return set_error(PBF_ERR_INVALID, "key %u needs more than %u bits", keys[i], key_bits);
    uint32_t *k = nullptr, *ka = nullptr, *ia = nullptr, *kb = nullptr, *ib = nullptr, *hist = nullptr, *tot = nullptr;
    int rc = PBF_OK;
    if ((rc = dalloc(k, n)) || (rc = dalloc(ka, n)) || (rc = dalloc(ia, n)) || (rc = dalloc(kb, n)) ||
        (rc = dalloc(ib, n)) || (rc = dalloc(hist, (size_t)256 * sort_num_tiles(n))) || (rc = dalloc(tot, 256))) {
        dfree(k); dfree(ka); dfree(ia); dfree(kb); dfree(ib); dfree(hist); dfree(tot);
        return rc;
    }
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    cudaMemcpyAsync(k, keys, 4 * (size_t)n, cudaMemcpyHostToDevice, st);
    uint32_t *ok = nullptr, *oi = nullptr;
    launch_radix_sort(n, key_bits, k, ka, ia, kb, ib, hist, tot, &ok, &oi, st, nullptr);
    cudaMemcpyAsync(sorted_keys, ok, 4 * (size_t)n, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(sorted_ids, oi, 4 * (size_t)n, cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    dfree(k); dfree(ka); dfree(ia); dfree(kb); dfree(ib); dfree(hist); dfree(tot);
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "sort_keys: %s", cudaGetErrorString(e));
    return PBF_OK;
}

extern "C" int pbf_build_table(const uint32_t* sorted_keys, uint32_t n, uint32_t hash_size, int32_t* table)
{
    if (!table || (n && !sorted_keys)) return set_error(PBF_ERR_INVALID, "null argument");
    if (hash_size == 0 || (hash_size & (hash_size - 1u))) return set_error(PBF_ERR_INVALID, "hash_size not a power of 2");
    for (uint32_t i = 0; i < n; ++i) {
        if (sorted_keys[i] >= hash_size) return set_error(PBF_ERR_INVALID, "key %u >= hash_size", sorted_keys[i]);
        if (i && sorted_keys[i] < sorted_keys[i - 1]) return set_error(PBF_ERR_INVALID, "keys not sorted at %u", i);
    }
    uint32_t* k = nullptr;
    int2* t = nullptr;
    int rc = PBF_OK;
    if ((n && (rc = dalloc(k, n))) || (rc = dalloc(t, hash_size))) {
        dfree(k); dfree(t);
        return rc;
    }
    cudaStream_t st;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (n) cudaMemcpyAsync(k, sorted_keys, 4 * (size_t)n, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(t, 0xFF, 8 * (size_t)hash_size, st);
    int sms = 148;
    if (n) launch_build_table(n, k, t, sms, st);
    cudaMemcpyAsync(table, t, 8 * (size_t)hash_size, cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    dfree(k); dfree(t);
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "build_table: %s", cudaGetErrorString(e));
    return PBF_OK;
}

// ---- timing / health ----------------------------------------------------------------------------
extern "C" int pbf_set_profiling(pbf_handle* h, int on)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    h->profiling = on != 0;
    return PBF_OK;
}

extern "C" int pbf_read_pass_times(pbf_handle* h, double* ms, uint64_t* cnt)
{
    CHECK_HANDLE(h);
    int rc = h->prof_collect();
    if (rc) return rc;
    for (int i = 0; i < PBF_NUM_PASS_SLOTS; ++i) {
        if (ms) ms[i] = h->prof_ms[i];
        if (cnt) cnt[i] = h->prof_count[i];
    }
    return PBF_OK;
}

extern "C" int pbf_reset_pass_times(pbf_handle* h)
{
    CHECK_HANDLE(h);
    int rc = h->prof_collect();
    if (rc) return rc;
    for (int i = 0; i < PBF_NUM_PASS_SLOTS; ++i) {
        h->prof_ms[i] = 0.0;
        h->prof_count[i] = 0;
    }
    return PBF_OK;
}

extern "C" int pbf_kernel_launches(pbf_handle* h, uint64_t* out)
{
    if (!h || !out) return set_error(PBF_ERR_INVALID, "null argument");
    *out = h->launches;
    return PBF_OK;
}

extern "C" int pbf_set_option(pbf_handle* h, int option, int value)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    switch (option) {
    case PBF_OPT_SPATIAL_ORDER:
        if (value != -1 && value != 4 && value != 8)
            return set_error(PBF_ERR_INVALID, "neighbour mode %d: -1 (automatic), 4 or 8", value);
        h->pass_mode = value;
        h->label_space = false;
        break;
    default: return set_error(PBF_ERR_INVALID, "unknown option %d", option);
    }
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_list_stats(pbf_handle* h, uint32_t* full_walks, uint32_t* bucket_walks, uint32_t* marked_buckets)
{
    CHECK_HANDLE(h);
    if (!full_walks || !bucket_walks || !marked_buckets) return set_error(PBF_ERR_INVALID, "null argument");
    *full_walks = *bucket_walks = *marked_buckets = 0;
    if (h->effective_mode() == 8) {
        // mode 8: particle passes that walked some rows through the hashed
        // buckets since the window was set up, particles of the last substep that moved beyond
        // the drift bound near a colliding cell and marked cells (counted per
        // pass), window cells that fail the collision test
        if (h->dflag) {
            uint32_t d3[3];
            CK(cudaMemcpyAsync(d3, h->dflag, sizeof(d3), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            *full_walks = d3[1];
            *bucket_walks = d3[0];
            *marked_buckets = d3[2];
        }
    }
    return PBF_OK;
}

extern "C" int pbf_set_use_graph(pbf_handle* h, int on)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    h->use_graph = on != 0;
    h->invalidate_graph();
    return PBF_OK;
}

extern "C" int pbf_check_finite(pbf_handle* h, uint32_t* bad)
{
    CHECK_HANDLE(h);
    if (!bad) return set_error(PBF_ERR_INVALID, "null argument");
    *bad = 0;
    if (h->n == 0) return PBF_OK;
    CK(cudaMemsetAsync(h->scalars + 1, 0, sizeof(uint32_t), h->stream));
    launch_check_finite(h->n, h->pos, h->vel, h->scalars + 1, h->num_sms, h->stream);
    ++h->launches;
    CK(cudaMemcpyAsync(bad, h->scalars + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return *bad ? set_error(PBF_ERR_NUMERIC, "%u particles hold NaN/Inf", *bad) : PBF_OK;
}
