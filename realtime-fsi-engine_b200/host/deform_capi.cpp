// deform_capi.cpp — C ABI of the host deformation solver (pbf_deform_*),
// the consumer of pbf_vertex_forces: a triangle mesh with rest positions,
// anchors, the Laplacian deformation and the per-frame handle driver.
#include <cstring>
#include <new>
#include <vector>

#include "../../include/deformation/LaplacianDeformation.h"
#include "../../include/pbf_b200.h"

namespace pbf {
int set_error(int code, const char* fmt, ...);
}

struct pbf_deform {
    pbfdrop::DeformMesh mesh;
    std::vector<pbfdrop::Vec3> rest;
    std::vector<int> lastHandles;
    pbfdrop::LaplacianDeformation* def = nullptr;
    ~pbf_deform() { delete def; }
};

using pbf::set_error;

extern "C" int pbf_deform_default_params(pbf_deform_params* p)
{
    if (!p) return set_error(PBF_ERR_INVALID, "null params");
    const pbfdrop::DeformParams d;
    p->stiffness = d.stiffness;
    p->max_displacement = d.maxDisplacement;
    p->max_total_disp = d.maxTotalDisp;
    p->restore_enabled = d.restoreEnabled ? 1u : 0u;
    p->restore_strength = d.restoreStrength;
    p->control_threshold = d.controlThreshold;
    p->control_threshold_low = d.controlThresholdLow;
    return PBF_OK;
}

extern "C" int pbf_deform_create(const double* verts3, int32_t nv, const int32_t* faces3, int32_t nf, pbf_deform** out)
{
    if (!out) return set_error(PBF_ERR_INVALID, "null output");
    *out = nullptr;
    if (!verts3 || !faces3 || nv < 3 || nf < 1) return set_error(PBF_ERR_INVALID, "bad mesh (nv=%d, nf=%d)", nv, nf);
    for (int32_t i = 0; i < 3 * nf; ++i)
        if (faces3[i] < 0 || faces3[i] >= nv) return set_error(PBF_ERR_INVALID, "face index %d out of range", faces3[i]);
    pbf_deform* d = new (std::nothrow) pbf_deform();
    if (!d) return set_error(PBF_ERR_ALLOC, "out of host memory");
    d->mesh.points.resize(nv);
    for (int32_t i = 0; i < nv; ++i) d->mesh.points[i] = {verts3[3 * i], verts3[3 * i + 1], verts3[3 * i + 2]};
    d->mesh.faces.resize(nf);
    for (int32_t f = 0; f < nf; ++f) d->mesh.faces[f] = {faces3[3 * f], faces3[3 * f + 1], faces3[3 * f + 2]};
    d->rest = d->mesh.points;
    d->def = new pbfdrop::LaplacianDeformation(d->mesh);
    d->def->initialize();
    *out = d;
    return PBF_OK;
}

extern "C" int pbf_deform_destroy(pbf_deform* d)
{
    delete d;
    return PBF_OK;
}

extern "C" int pbf_deform_set_mode(pbf_deform* d, int32_t use_local, int32_t kring, int32_t use_incremental)
{
    if (!d) return set_error(PBF_ERR_INVALID, "null deformer");
    if (kring < 0) return set_error(PBF_ERR_INVALID, "k-ring %d < 0", kring);
    d->def->setUseLocal(use_local != 0);
    d->def->setLocalKRing(kring);
    d->def->setUseIncremental(use_incremental != 0);
    return PBF_OK;
}

extern "C" int pbf_deform_add_anchor(pbf_deform* d, int32_t v)
{
    if (!d) return set_error(PBF_ERR_INVALID, "null deformer");
    if (v < 0 || v >= (int32_t)d->mesh.points.size()) return set_error(PBF_ERR_INVALID, "vertex %d out of range", v);
    d->def->addAnchor(v);
    return PBF_OK;
}

extern "C" int pbf_deform_set_control_points(pbf_deform* d, const int32_t* idx, const double* targets3, int32_t n)
{
    if (!d) return set_error(PBF_ERR_INVALID, "null deformer");
    if (n < 0 || (n > 0 && (!idx || !targets3))) return set_error(PBF_ERR_INVALID, "bad control points");
    std::vector<int> iv(n);
    std::vector<pbfdrop::Vec3> tv(n);
    for (int32_t i = 0; i < n; ++i) {
        if (idx[i] < 0 || idx[i] >= (int32_t)d->mesh.points.size())
            return set_error(PBF_ERR_INVALID, "vertex %d out of range", idx[i]);
        iv[i] = idx[i];
        tv[i] = {targets3[3 * i], targets3[3 * i + 1], targets3[3 * i + 2]};
    }
    d->def->setControlPoints(iv, tv);
    return PBF_OK;
}

extern "C" int pbf_deform_precompute(pbf_deform* d)
{
    if (!d) return set_error(PBF_ERR_INVALID, "null deformer");
    d->def->precomputeSystem();
    return PBF_OK;
}

extern "C" int pbf_deform_solve(pbf_deform* d)
{
    if (!d) return set_error(PBF_ERR_INVALID, "null deformer");
    d->def->solve();
    return PBF_OK;
}

extern "C" int pbf_deform_vertices(pbf_deform* d, double* out3, int32_t nv)
{
    if (!d || !out3) return set_error(PBF_ERR_INVALID, "null argument");
    if (nv != (int32_t)d->mesh.points.size()) return set_error(PBF_ERR_INVALID, "nv=%d, mesh has %zu", nv, d->mesh.points.size());
    for (int32_t i = 0; i < nv; ++i)
        for (int a = 0; a < 3; ++a) out3[3 * i + a] = d->mesh.points[i][a];
    return PBF_OK;
}

extern "C" int pbf_deform_set_vertices(pbf_deform* d, const double* v3, int32_t nv)
{
    if (!d || !v3) return set_error(PBF_ERR_INVALID, "null argument");
    if (nv != (int32_t)d->mesh.points.size()) return set_error(PBF_ERR_INVALID, "nv=%d, mesh has %zu", nv, d->mesh.points.size());
    for (int32_t i = 0; i < nv; ++i) d->mesh.points[i] = {v3[3 * i], v3[3 * i + 1], v3[3 * i + 2]};
    return PBF_OK;
}

extern "C" int pbf_deform_step(pbf_deform* d, const float* forces3, int32_t nv, float dt, const pbf_deform_params* p,
                               int32_t* handle_count, int32_t* refactored, int32_t* moved)
{
    if (!d || !forces3 || !p) return set_error(PBF_ERR_INVALID, "null argument");
    if (nv != (int32_t)d->mesh.points.size()) return set_error(PBF_ERR_INVALID, "nv=%d, mesh has %zu", nv, d->mesh.points.size());
    std::vector<pbfdrop::Vec3> f(nv);
    for (int32_t i = 0; i < nv; ++i) f[i] = {forces3[3 * i], forces3[3 * i + 1], forces3[3 * i + 2]};
    pbfdrop::DeformParams prm;
    prm.stiffness = p->stiffness;
    prm.maxDisplacement = p->max_displacement;
    prm.maxTotalDisp = p->max_total_disp;
    prm.restoreEnabled = p->restore_enabled != 0;
    prm.restoreStrength = p->restore_strength;
    prm.controlThreshold = p->control_threshold;
    prm.controlThresholdLow = p->control_threshold_low;
    int hc = 0;
    bool rf = false;
    const bool mv = d->def->deformStep(f, dt, prm, d->rest, d->lastHandles, &hc, &rf);
    if (handle_count) *handle_count = hc;
    if (refactored) *refactored = rf ? 1 : 0;
    if (moved) *moved = mv ? 1 : 0;
    return PBF_OK;
}

extern "C" int pbf_deform_patch_size(pbf_deform* d, int32_t* size)
{
    if (!d || !size) return set_error(PBF_ERR_INVALID, "null argument");
    *size = d->def->getLocalPatchSize();
    return PBF_OK;
}

extern "C" int pbf_deform_verify_incremental(pbf_deform* d, double* max_diff)
{
    if (!d || !max_diff) return set_error(PBF_ERR_INVALID, "null argument");
    *max_diff = d->def->verifyIncremental();
    return PBF_OK;
}
