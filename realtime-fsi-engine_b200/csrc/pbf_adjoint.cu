// pbf_adjoint.cu — differentiable step of the multi-scene engine.
//
// pbf_batch_forward_record runs one step (every substep, then vorticity)
// exactly as pbf_batch_step does, saving the particle state at the start of
// each substep.  pbf_batch_backward then walks the substeps in reverse: it
// recomputes the substep from its checkpoint (predict, segmented sort, cell
// table, reorder, processing order — the permutation is replayed, not
// differentiated), re-runs the solver iterations recording (x*, lambda), the
// lambda denominators and the raw dp of every iteration, and runs the
// reverse kernels of k_adjoint.cu: vorticity (last substep), integrate,
// (deltaP+apply, lambda) per iteration, predict.  Gradients are with respect
// to the initial positions and velocities and each scene's SDF translation.
// Both sequences are captured once into CUDA graphs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "../../include/pbf_b200.h"
#include "pbf_batch.h"
#include "pbf_engine.h"

using namespace pbf;

#define ACK(call)                                                                                  \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

template <class T>
static int aalloc(T*& p, size_t count)
{
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        return set_error(PBF_ERR_ALLOC, "cudaMalloc(%zu B): %s", count * sizeof(T), cudaGetErrorString(e));
    }
    return PBF_OK;
}

template <class T>
static void afree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

void pbf_batch::ad_free()
{
    afree(cp_pos); afree(cp_vel); afree(xl); afree(auxl); afree(auxd); afree(rhol);
    afree(gxa); afree(gxb); afree(gv); afree(x0b); afree(pb); afree(vb); afree(pbs); afree(omb);
    afree(tpos); afree(tvel); afree(tgrad);
    ad_subs = ad_iters = 0;
    recorded = false;
}

int pbf_batch::ad_alloc()
{
    const uint32_t S = cfg.substep_iterations, I = cfg.solver_iterations;
    if (S == ad_subs && I == ad_iters && cp_pos) return PBF_OK;
    ad_free();
    const size_t c = std::max<uint32_t>(n, 1u);
    int rc;
    if ((rc = aalloc(cp_pos, c * S)) || (rc = aalloc(cp_vel, c * S)) || (rc = aalloc(xl, c * std::max(I, 1u))) ||
        (rc = aalloc(auxl, c * std::max(I, 1u))) || (rc = aalloc(auxd, c * std::max(I, 1u))) ||
        (rc = aalloc(rhol, c * std::max(I, 1u))) || (rc = aalloc(gxa, c)) || (rc = aalloc(gxb, c)) ||
        (rc = aalloc(gv, c)) || (rc = aalloc(x0b, c)) || (rc = aalloc(pb, c)) || (rc = aalloc(vb, c)) ||
        (rc = aalloc(pbs, c)) || (rc = aalloc(omb, c)) || (rc = aalloc(tpos, c)) || (rc = aalloc(tvel, c)) ||
        (rc = aalloc(tgrad, 4 * scenes.size()))) {
        ad_free();
        return rc;
    }
    ad_subs = S;
    ad_iters = I;
    return PBF_OK;
}

int pbf_batch::record_body()
{
    const DevParams P = dev_params();
    BatchLaunch L = launch;
    L.sms = num_sms;
    for (uint32_t sub = 0; sub < cfg.substep_iterations; ++sub) {
        ACK(cudaMemcpyAsync(cp_pos + (size_t)sub * n, pos, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
        ACK(cudaMemcpyAsync(cp_vel + (size_t)sub * n, vel, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
        const int rc = substep_body(pos, vel, pos, vel);
        if (rc) return rc;
    }
    if (cfg.enable_vorticity) {
        launch_b_vorticity(P, L, scenes_dev, scene_of, sx0, somega, ids, vel, table, order, stream);
        ++launches;
    }
    return PBF_OK;
}

// Inputs: pb, vb (adjoints of the recorded step's final state).  Outputs:
// pb, vb (adjoints of its initial state), tgrad (of the SDF translations).
int pbf_batch::backward_body()
{
    const DevParams P = dev_params();
    BatchLaunch L = launch;
    L.sms = num_sms;
    const int sms = num_sms;
    const uint32_t S = cfg.substep_iterations, I = cfg.solver_iterations;
    const bool vort = cfg.enable_vorticity != 0;
    ACK(cudaMemsetAsync(tgrad, 0, sizeof(float) * 4 * scenes.size(), stream));
    ACK(cudaMemsetAsync(pbs, 0, sizeof(float4) * n, stream));
    ACK(cudaMemsetAsync(omb, 0, sizeof(float4) * n, stream));
    for (int sub = (int)S - 1; sub >= 0; --sub) {
        const float4* src_pos = cp_pos + (size_t)sub * n;
        const float4* src_vel = cp_vel + (size_t)sub * n;
        // replay the substep's sort, table and processing order
        launch_b_predict(P, scenes_dev, scene_of, src_pos, src_vel, keys, sms, stream);
        launch_radix_sort(n, key_bits, keys, ka, ia, kb, ib, hist, totals, &skeys, &ids, stream, &launches);
        ACK(cudaMemsetAsync(table, 0xFF, sizeof(int2) * (size_t)table_size, stream));
        launch_build_table(n, skeys, table, sms, stream);
        launch_b_reorder(P, scenes_dev, scene_of, ids, src_pos, src_vel, sx[0], sv, sx0, lod,
                         morton ? mcode : nullptr, mbits, sms, stream);
        launches += 3;
        order = nullptr;
        if (morton) {
            uint32_t* msorted = nullptr;
            launch_radix_sort(n, order_bits, mcode, mka, mia, mkb, mib, hist, totals, &msorted, &order, stream,
                              &launches);
        }
        // recompute the iterations, recording what the reverse reads
        for (uint32_t it = 1; it <= I; ++it) {
            float4* xli = xl + (size_t)(it - 1) * n;
            launch_ad_lambda_rec(P, scenes_dev, scene_of, order, table, sx[0], xli, auxl + (size_t)(it - 1) * n,
                                 rhol + (size_t)(it - 1) * n, stream);
            launch_ad_deltap_rec(P, scenes_dev, scene_of, order, table, xli, sx[0], auxd + (size_t)(it - 1) * n,
                                 stream);
            launches += 2;
        }
        const bool last = (sub == (int)S - 1) && vort;
        if (last) {
            // committed state and omega of the last substep, for the vorticity reverse
            launch_b_integrate(P, L, scenes_dev, scene_of, sx[0], sv, sx0, somega, ids, tpos, tvel, table, order,
                               stream);
            launch_ad_vorticity(P, scenes_dev, scene_of, order, table, sx0, somega, ids, vb, pbs, omb, stream);
            launches += 2;
        }
        ACK(cudaMemsetAsync(gxa, 0, sizeof(float4) * n, stream));
        ACK(cudaMemsetAsync(gxb, 0, sizeof(float4) * n, stream));
        ACK(cudaMemsetAsync(gv, 0, sizeof(float4) * n, stream));
        launch_ad_integrate(P, scenes_dev, scene_of, order, table, sx[0], sv, src_pos, ids, pb, vb,
                            last ? pbs : nullptr, last ? omb : nullptr, somega, gxa, gv, x0b, tgrad, stream);
        ++launches;
        float4* a = gxa;
        float4* b = gxb;
        for (int it = (int)I; it >= 1; --it) {
            const float4* xli = xl + (size_t)(it - 1) * n;
            launch_ad_deltap(P, scenes_dev, scene_of, order, table, xli, auxd + (size_t)(it - 1) * n, a, b, tgrad,
                             stream);
            launch_ad_lambda(P, scenes_dev, scene_of, order, table, xli, auxl + (size_t)(it - 1) * n,
                             rhol + (size_t)(it - 1) * n, b, stream);
            launches += 2;
            ACK(cudaMemsetAsync(a, 0, sizeof(float4) * n, stream));
            std::swap(a, b);
        }
        launch_ad_predict(n, P.dt, ids, a, gv, x0b, pb, vb, sms, stream);
        ++launches;
    }
    return PBF_OK;
}

// Run body() once, through a graph captured on first use when enabled.
template <class Body>
static int run_graph(pbf_batch* b, cudaGraph_t& g, cudaGraphExec_t& ex, uint64_t& glaunches, Body body)
{
    if (!b->use_graph) return body();
    if (!ex) {
        const uint64_t before = b->launches;
        b->capturing = true;
        ACK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = body();
        cudaGraph_t gg = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &gg);
        b->capturing = false;
        if (rc) {
            if (gg) cudaGraphDestroy(gg);
            return rc;
        }
        if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
        g = gg;
        ACK(cudaGraphInstantiate(&ex, g, 0));
        glaunches = b->launches - before;
        b->launches = before;
    }
    ACK(cudaGraphLaunch(ex, b->stream));
    b->launches += glaunches;
    return PBF_OK;
}

static int check_differentiable(const pbf_batch* b)
{
    if (b->cfg.enable_apbf) return set_error(PBF_ERR_STATE, "the adjoint needs APBF off");
    if (b->n == 0) return set_error(PBF_ERR_STATE, "empty batch");
    return PBF_OK;
}

// ---- C ABI --------------------------------------------------------------------------------
#define CHECK_B(b)                                                                                 \
    do {                                                                                           \
        if (!(b)) return pbf::set_error(PBF_ERR_INVALID, "null batch");                            \
        cudaError_t e_ = cudaSetDevice((b)->device);                                               \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e_));      \
    } while (0)

extern "C" int pbf_batch_set_sdf_offset(pbf_batch* b, uint32_t scene, const float t[3])
{
    CHECK_B(b);
    if (scene >= b->scenes.size()) return set_error(PBF_ERR_INVALID, "scene %u out of range", scene);
    if (!t) return set_error(PBF_ERR_INVALID, "null offset");
    for (int a = 0; a < 3; ++a) b->scenes[scene].sdf_offset[a] = t[a];
    b->recorded = false;
    return b->upload_scenes();
}

extern "C" int pbf_batch_set_state(pbf_batch* b, const void* pos4, const void* vel4)
{
    CHECK_B(b);
    if (b->n == 0) return PBF_OK;
    if (!pos4 || !vel4) return set_error(PBF_ERR_INVALID, "null state");
    ACK(cudaMemcpyAsync(b->pos, pos4, sizeof(float4) * b->n, cudaMemcpyDefault, b->stream));
    ACK(cudaMemcpyAsync(b->vel, vel4, sizeof(float4) * b->n, cudaMemcpyDefault, b->stream));
    ACK(cudaStreamSynchronize(b->stream));
    b->recorded = false;
    return PBF_OK;
}

extern "C" int pbf_batch_get_state(pbf_batch* b, void* pos4, void* vel4)
{
    CHECK_B(b);
    if (b->n == 0) return PBF_OK;
    if (pos4) ACK(cudaMemcpyAsync(pos4, b->pos, sizeof(float4) * b->n, cudaMemcpyDefault, b->stream));
    if (vel4) ACK(cudaMemcpyAsync(vel4, b->vel, sizeof(float4) * b->n, cudaMemcpyDefault, b->stream));
    ACK(cudaStreamSynchronize(b->stream));
    return PBF_OK;
}

extern "C" int pbf_batch_forward_record(pbf_batch* b)
{
    CHECK_B(b);
    int rc = check_differentiable(b);
    if (rc) return rc;
    if ((rc = b->ad_alloc())) return rc;
    rc = run_graph(b, b->rec_graph, b->rec_exec, b->rec_launches, [&] { return b->record_body(); });
    if (rc) return rc;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    b->recorded = true;
    return PBF_OK;
}

extern "C" int pbf_batch_backward(pbf_batch* b, const void* gpos4, const void* gvel4, void* out_gpos4,
                                  void* out_gvel4, float* out_gt)
{
    CHECK_B(b);
    int rc = check_differentiable(b);
    if (rc) return rc;
    if (!b->recorded) return set_error(PBF_ERR_STATE, "backward without a recorded forward");
    const size_t bytes = sizeof(float4) * b->n;
    if (gpos4) ACK(cudaMemcpyAsync(b->pb, gpos4, bytes, cudaMemcpyDefault, b->stream));
    else ACK(cudaMemsetAsync(b->pb, 0, bytes, b->stream));
    if (gvel4) ACK(cudaMemcpyAsync(b->vb, gvel4, bytes, cudaMemcpyDefault, b->stream));
    else ACK(cudaMemsetAsync(b->vb, 0, bytes, b->stream));
    rc = run_graph(b, b->bwd_graph, b->bwd_exec, b->bwd_launches, [&] { return b->backward_body(); });
    if (rc) return rc;
    if (out_gpos4) ACK(cudaMemcpyAsync(out_gpos4, b->pb, bytes, cudaMemcpyDefault, b->stream));
    if (out_gvel4) ACK(cudaMemcpyAsync(out_gvel4, b->vb, bytes, cudaMemcpyDefault, b->stream));
    if (out_gt) {
        std::vector<float> t(4 * b->scenes.size());
        ACK(cudaMemcpyAsync(t.data(), b->tgrad, sizeof(float) * t.size(), cudaMemcpyDeviceToHost, b->stream));
        ACK(cudaStreamSynchronize(b->stream));
        for (size_t k = 0; k < b->scenes.size(); ++k)
            for (int a = 0; a < 3; ++a) out_gt[3 * k + a] = t[4 * k + a];
    }
    ACK(cudaStreamSynchronize(b->stream));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "kernel launch: %s", cudaGetErrorString(e));
    return PBF_OK;
}
