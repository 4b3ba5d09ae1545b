// pbf_mesh.cu — triangle-mesh SDF entry points of the C ABI.
//
// pbf_set_sdf_mesh      = SDFBoundary::buildFromMesh   (SDFBoundary.cpp:278-398)
// pbf_rebuild_mesh      = buildFromMesh again for moved vertices of the same faces
// pbf_update_mesh_vertices = SDFBoundary::refitFromMesh (SDFBoundary.cpp:455-465)
// pbf_closest_triangle  = SDFBoundary::closestTriangle  (SDFBoundary.cpp:600-610)
// pbf_vertex_forces     = computeContactForces          (src/main.cpp:604-710)
//
// The host derives only what depends on the face list: per-vertex (face,
// corner) lists and each face edge's partner face (integer adjacency, once per
// face list), and the grid geometry (origin = bbox - 5 cells, dims =
// ceil(span / cell)) from the vertex bounding box.  Everything that depends
// on vertex positions runs on the GPU: the LBVH build and refit, face normals,
// the angle-weighted vertex and edge pseudo-normals, the distance grid and the
// forces.  A build computes the pseudo-normals; a refit keeps them, as the
// reference does (SDFBoundary.h:58-62).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/pbf_b200.h"
#include "pbf_engine.h"
#include "pbf_kernels.h"

using namespace pbf;

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return pbf::set_error(PBF_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

namespace {

struct MeshHost {
    std::vector<int3> faces;
    std::vector<float3> verts_f;
    // face-list adjacency (see build_adjacency)
    int* d_voff = nullptr;
    int2* d_vfc = nullptr;
    int* d_partner = nullptr;
    // device allocations
    int3* d_faces = nullptr;
    float3* d_verts = nullptr;
    float3* d_face_n = nullptr;
    float3* d_edge_n = nullptr;
    float3* d_vert_n = nullptr;
    int2* d_child = nullptr;
    int* d_parent = nullptr;
    float4* d_bmin = nullptr;
    float4* d_bmax = nullptr;
    int* d_leaf_face = nullptr;
    uint32_t* d_flags = nullptr;
    uint32_t *d_codes = nullptr, *d_ka = nullptr, *d_ia = nullptr, *d_kb = nullptr, *d_ib = nullptr;
    uint32_t *d_hist = nullptr, *d_tot = nullptr;
    int* d_frontier = nullptr;
};

struct D3 {
    double x, y, z;
};

template <class T>
void dfree(T*& p)
{
    if (p) cudaFree(p);
    p = nullptr;
}

template <class T>
int dalloc(T*& p, size_t n)
{
    dfree(p);
    if (n == 0) return PBF_OK;
    const cudaError_t e = cudaMalloc((void**)&p, n * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        return set_error(PBF_ERR_ALLOC, "cudaMalloc(%zu B): %s", n * sizeof(T), cudaGetErrorString(e));
    }
    return PBF_OK;
}

void free_mesh_host(MeshHost* m)
{
    if (!m) return;
    dfree(m->d_faces); dfree(m->d_verts); dfree(m->d_face_n); dfree(m->d_edge_n); dfree(m->d_vert_n);
    dfree(m->d_child); dfree(m->d_parent); dfree(m->d_bmin); dfree(m->d_bmax); dfree(m->d_leaf_face);
    dfree(m->d_flags); dfree(m->d_codes); dfree(m->d_ka); dfree(m->d_ia); dfree(m->d_kb); dfree(m->d_ib);
    dfree(m->d_hist); dfree(m->d_tot); dfree(m->d_frontier);
    dfree(m->d_voff); dfree(m->d_vfc); dfree(m->d_partner);
    delete m;
}

// kMeshFrontier subtrees that together cover the tree (internal nodes [0,
// nf-1), leaves [nf-1, 2nf-1)): starting from the root, the internal node
// with the most leaves is replaced by its two children until there are
// kMeshFrontier subtrees or only leaves; unused entries are -1.
std::vector<int> mesh_frontier(const std::vector<int2>& child, int nf)
{
    std::vector<int> fr(kMeshFrontier, -1);
    const int n_int = nf - 1;
    fr[0] = 0;
    if (n_int <= 0) return fr;
    const int nodes = 2 * nf - 1;
    std::vector<int> leaves(n_int, 0), order;
    order.reserve(n_int);
    std::vector<int> st{0};
    while (!st.empty() && (int)order.size() < n_int) {
        const int u = st.back();
        st.pop_back();
        order.push_back(u);
        for (const int c : {child[u].x, child[u].y})
            if (c >= 0 && c < n_int) st.push_back(c);
    }
    auto count = [&](int c) { return c >= n_int && c < nodes ? 1 : (c >= 0 && c < n_int ? leaves[c] : 0); };
    for (auto it = order.rbegin(); it != order.rend(); ++it) leaves[*it] = count(child[*it].x) + count(child[*it].y);
    int used = 1;
    while (used < kMeshFrontier) {
        int j = -1;
        for (int k = 0; k < used; ++k)
            if (fr[k] < n_int && (j < 0 || leaves[fr[k]] > leaves[fr[j]])) j = k;
        if (j < 0) break;
        const int2 ch = child[fr[j]];
        fr[j] = ch.x;
        fr[used++] = ch.y;
    }
    return fr;
}

// Adjacency of a face list (SDFBoundary.cpp:341-383 walks the same
// relations): for every vertex its (face, corner) incidences in ascending
// face order, and for every face edge slot (AB, AC, BC) the other face of an
// edge that exactly two face slots share (-1 otherwise).  The slot an edge
// lands in follows the reference's test order: AB if it matches, else AC,
// else BC.
void build_adjacency(const int32_t* faces, int32_t nv, int32_t nf, std::vector<int>& voff, std::vector<int2>& vfc,
                     std::vector<int>& partner)
{
    voff.assign((size_t)nv + 1, 0);
    for (int64_t i = 0; i < 3 * (int64_t)nf; ++i) ++voff[(size_t)faces[i] + 1];
    for (int32_t v = 0; v < nv; ++v) voff[(size_t)v + 1] += voff[(size_t)v];
    vfc.resize(3 * (size_t)nf);
    std::vector<int> cur(voff.begin(), voff.end() - 1);
    for (int32_t f = 0; f < nf; ++f)
        for (int c = 0; c < 3; ++c) vfc[(size_t)cur[(size_t)faces[3 * f + c]]++] = make_int2(f, c);
    struct E {
        int a, b, t;
    };
    std::vector<E> edges;
    edges.reserve(3 * (size_t)nf);
    for (int32_t f = 0; f < nf; ++f) {
        const int A = faces[3 * f], B = faces[3 * f + 1], C = faces[3 * f + 2];
        edges.push_back({std::min(A, B), std::max(A, B), f});
        edges.push_back({std::min(A, C), std::max(A, C), f});
        edges.push_back({std::min(B, C), std::max(B, C), f});
    }
    std::sort(edges.begin(), edges.end(), [](const E& x, const E& y) {
        return x.a != y.a ? x.a < y.a : (x.b != y.b ? x.b < y.b : x.t < y.t);
    });
    partner.assign(3 * (size_t)nf, -1);
    for (size_t i = 0; i < edges.size();) {
        size_t j = i;
        while (j < edges.size() && edges[j].a == edges[i].a && edges[j].b == edges[i].b) ++j;
        if (j - i == 2) {
            for (size_t k = i; k < j; ++k) {
                const int t = edges[k].t, a = edges[k].a, b = edges[k].b;
                const int A = faces[3 * t], B = faces[3 * t + 1], C = faces[3 * t + 2];
                const int slot = (std::min(A, B) == a && std::max(A, B) == b)   ? 0
                                 : (std::min(A, C) == a && std::max(A, C) == b) ? 1
                                                                                : 2;
                partner[3 * (size_t)t + slot] = edges[k == i ? i + 1 : i].t;
            }
        }
        i = j;
    }
}

}  // namespace

void pbf_handle::mesh_free()
{
    free_mesh_host(static_cast<MeshHost*>(mesh_host));
    mesh_host = nullptr;
    mesh = MeshDev{};
    mesh_attached = false;
    if (force_acc) cudaFree(force_acc);
    if (force_contacts) cudaFree(force_contacts);
    if (force_out) cudaFree(force_out);
    force_acc = nullptr;
    force_contacts = nullptr;
    force_out = nullptr;
}

static int validate_mesh(const double* verts, int32_t nv, const int32_t* faces, int32_t nf)
{
    if (!verts || !faces || nv <= 0 || nf <= 0) return set_error(PBF_ERR_INVALID, "empty mesh");
    for (int64_t i = 0; i < 3 * (int64_t)nf; ++i)
        if (faces[i] < 0 || faces[i] >= nv) return set_error(PBF_ERR_INVALID, "face index %d out of range", faces[i]);
    for (int64_t i = 0; i < 3 * (int64_t)nv; ++i)
        if (!std::isfinite(verts[i])) return set_error(PBF_ERR_INVALID, "non-finite vertex coordinate");
    return PBF_OK;
}

// Everything of a build that depends on vertex positions, for the face list
// already on the device: grid geometry from the bounding box
// (SDFBoundary.cpp:291-308), the LBVH over Morton codes of the face
// centroids, its subtree frontier, node boxes and face normals, the vertex
// and edge pseudo-normals, the distance grid.
static int mesh_build_geometry(pbf_handle* h, const double* verts, double cell)
{
    MeshHost* m = static_cast<MeshHost*>(h->mesh_host);
    MeshDev& M = h->mesh;
    const int nv = M.nv, nf = M.nf;
    D3 bmin{1e30, 1e30, 1e30}, bmax{-1e30, -1e30, -1e30};
    for (int i = 0; i < nv; ++i) {
        bmin = {std::min(bmin.x, verts[3 * i]), std::min(bmin.y, verts[3 * i + 1]), std::min(bmin.z, verts[3 * i + 2])};
        bmax = {std::max(bmax.x, verts[3 * i]), std::max(bmax.y, verts[3 * i + 1]), std::max(bmax.z, verts[3 * i + 2])};
    }
    const double buffer = cell * 5.0;
    const double o[3] = {bmin.x - buffer, bmin.y - buffer, bmin.z - buffer};
    const double span[3] = {(bmax.x + buffer) - o[0], (bmax.y + buffer) - o[1], (bmax.z + buffer) - o[2]};
    int32_t dims[3];
    for (int a = 0; a < 3; ++a) dims[a] = (int32_t)std::ceil(span[a] / cell);
    const size_t total = (size_t)dims[0] * dims[1] * dims[2];
    if (total == 0 || total > ((size_t)1 << 31)) return set_error(PBF_ERR_INVALID, "SDF grid of %zu voxels", total);

    for (int i = 0; i < nv; ++i)
        m->verts_f[i] = make_float3((float)verts[3 * i], (float)verts[3 * i + 1], (float)verts[3 * i + 2]);
    cudaStream_t st = h->stream;
    CK(cudaMemcpyAsync(m->d_verts, m->verts_f.data(), sizeof(float3) * nv, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(m->d_parent, 0xFF, sizeof(int) * (2 * (size_t)nf - 1), st));

    // LBVH: Morton codes of the face centroids over the vertex bbox
    const float3 lo = make_float3((float)bmin.x, (float)bmin.y, (float)bmin.z);
    const double ex = std::max(bmax.x - bmin.x, 1e-30), ey = std::max(bmax.y - bmin.y, 1e-30),
                 ez = std::max(bmax.z - bmin.z, 1e-30);
    const float3 inv_ext = make_float3((float)(1.0 / ex), (float)(1.0 / ey), (float)(1.0 / ez));
    launch_morton(nf, m->d_faces, m->d_verts, lo, inv_ext, m->d_codes, st);
    uint32_t *sk = nullptr, *sid = nullptr;
    launch_radix_sort((uint32_t)nf, 30, m->d_codes, m->d_ka, m->d_ia, m->d_kb, m->d_ib, m->d_hist, m->d_tot, &sk,
                      &sid, st, &h->launches);
    CK(cudaMemcpyAsync(m->d_leaf_face, sid, sizeof(int) * nf, cudaMemcpyDeviceToDevice, st));
    launch_lbvh_topology(nf, sk, m->d_child, m->d_parent, st);
    h->launches += 2;
    {
        // the grid kernel's per-lane subtrees (the tree shape is fixed until the next build)
        std::vector<int2> child(std::max(1, nf - 1), make_int2(-1, -1));
        if (nf > 1)
            CK(cudaMemcpyAsync(child.data(), m->d_child, sizeof(int2) * (size_t)(nf - 1), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const std::vector<int> fr = mesh_frontier(child, nf);
        CK(cudaMemcpyAsync(m->d_frontier, fr.data(), sizeof(int) * kMeshFrontier, cudaMemcpyHostToDevice, st));
    }
    launch_mesh_refit(M, st, &h->launches);
    launch_mesh_pseudo_normals(M, m->d_voff, m->d_vfc, m->d_partner, m->d_vert_n, m->d_edge_n, st, &h->launches);

    for (int a = 0; a < 3; ++a) h->origin_d[a] = o[a];
    h->cell_d = cell;
    const float of[3] = {(float)o[0], (float)o[1], (float)o[2]};
    int rc;
    if ((rc = h->upload_grid(nullptr, dims, of, (float)cell))) return rc;
    launch_mesh_grid_d(M, dims[0], dims[1], dims[2], h->origin_d, cell, h->grid, h->num_sms, st);
    launch_sdf_slab_min(h->grid, dims[0], dims[1], dims[2], h->slab_min, st);
    h->launches += 2;
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return PBF_OK;
}

extern "C" int pbf_set_sdf_mesh(pbf_handle* h, const double* verts, int32_t nv, const int32_t* faces, int32_t nf,
                                double cell)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    CK(cudaSetDevice(h->device));
    int rc = validate_mesh(verts, nv, faces, nf);
    if (rc) return rc;
    if (!(cell > 0.0)) return set_error(PBF_ERR_INVALID, "cell size must be > 0");
    CK(cudaStreamSynchronize(h->stream));
    h->mesh_free();

    std::vector<int> voff, partner;
    std::vector<int2> vfc;
    build_adjacency(faces, nv, nf, voff, vfc, partner);

    MeshHost* m = new MeshHost();
    h->mesh_host = m;
    m->faces.resize(nf);
    for (int f = 0; f < nf; ++f) m->faces[f] = make_int3(faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]);
    m->verts_f.resize(nv);

    const size_t nodes = 2 * (size_t)nf - 1;
    if ((rc = dalloc(m->d_faces, nf)) || (rc = dalloc(m->d_verts, nv)) || (rc = dalloc(m->d_face_n, nf)) ||
        (rc = dalloc(m->d_edge_n, 3 * (size_t)nf)) || (rc = dalloc(m->d_vert_n, nv)) ||
        (rc = dalloc(m->d_child, std::max<size_t>(1, nf - 1))) || (rc = dalloc(m->d_parent, nodes)) ||
        (rc = dalloc(m->d_bmin, nodes)) || (rc = dalloc(m->d_bmax, nodes)) || (rc = dalloc(m->d_leaf_face, nf)) ||
        (rc = dalloc(m->d_flags, std::max<size_t>(1, nf - 1))) || (rc = dalloc(m->d_codes, nf)) ||
        (rc = dalloc(m->d_ka, nf)) || (rc = dalloc(m->d_ia, nf)) || (rc = dalloc(m->d_kb, nf)) ||
        (rc = dalloc(m->d_ib, nf)) || (rc = dalloc(m->d_hist, (size_t)256 * sort_num_tiles(nf))) ||
        (rc = dalloc(m->d_tot, 256)) || (rc = dalloc(m->d_frontier, (size_t)kMeshFrontier)) ||
        (rc = dalloc(m->d_voff, (size_t)nv + 1)) || (rc = dalloc(m->d_vfc, 3 * (size_t)nf)) ||
        (rc = dalloc(m->d_partner, 3 * (size_t)nf)) || (rc = dalloc(h->force_acc, 3 * (size_t)nv)) ||
        (rc = dalloc(h->force_contacts, 1)) || (rc = dalloc(h->force_out, 3 * (size_t)nv))) {
        h->mesh_free();
        return rc;
    }
    cudaStream_t st = h->stream;
    CK(cudaMemcpyAsync(m->d_faces, m->faces.data(), sizeof(int3) * nf, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(m->d_voff, voff.data(), sizeof(int) * voff.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(m->d_vfc, vfc.data(), sizeof(int2) * vfc.size(), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(m->d_partner, partner.data(), sizeof(int) * partner.size(), cudaMemcpyHostToDevice, st));

    MeshDev M{};
    M.nv = nv;
    M.nf = nf;
    M.faces = m->d_faces;
    M.verts = m->d_verts;
    M.face_n = m->d_face_n;
    M.edge_n = m->d_edge_n;
    M.vert_n = m->d_vert_n;
    M.child = m->d_child;
    M.parent = m->d_parent;
    M.bmin = m->d_bmin;
    M.bmax = m->d_bmax;
    M.leaf_face = m->d_leaf_face;
    M.flags = m->d_flags;
    M.frontier = m->d_frontier;
    h->mesh = M;
    if ((rc = mesh_build_geometry(h, verts, cell))) {
        h->mesh_free();
        return rc;
    }
    h->mesh_attached = true;
    return PBF_OK;
}

extern "C" int pbf_rebuild_mesh(pbf_handle* h, const double* verts, int32_t nv)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    CK(cudaSetDevice(h->device));
    if (!h->mesh_attached) return set_error(PBF_ERR_STATE, "no mesh attached");
    if (!verts || nv != h->mesh.nv) return set_error(PBF_ERR_INVALID, "vertex count %d != %d", nv, h->mesh.nv);
    for (int64_t i = 0; i < 3 * (int64_t)nv; ++i)
        if (!std::isfinite(verts[i])) return set_error(PBF_ERR_INVALID, "non-finite vertex coordinate");
    CK(cudaStreamSynchronize(h->stream));
    return mesh_build_geometry(h, verts, h->cell_d);
}

extern "C" int pbf_update_mesh_vertices(pbf_handle* h, const double* verts, int32_t nv)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    CK(cudaSetDevice(h->device));
    if (!h->mesh_attached) return set_error(PBF_ERR_STATE, "no mesh attached");
    if (!verts || nv != h->mesh.nv) return set_error(PBF_ERR_INVALID, "vertex count %d != %d", nv, h->mesh.nv);
    MeshHost* m = static_cast<MeshHost*>(h->mesh_host);
    for (int i = 0; i < nv; ++i) {
        if (!std::isfinite(verts[3 * i]) || !std::isfinite(verts[3 * i + 1]) || !std::isfinite(verts[3 * i + 2]))
            return set_error(PBF_ERR_INVALID, "non-finite vertex %d", i);
        m->verts_f[i] = make_float3((float)verts[3 * i], (float)verts[3 * i + 1], (float)verts[3 * i + 2]);
    }
    cudaStream_t st = h->stream;
    CK(cudaMemcpyAsync(m->d_verts, m->verts_f.data(), sizeof(float3) * nv, cudaMemcpyHostToDevice, st));
    launch_mesh_refit(h->mesh, st, &h->launches);
    launch_mesh_grid_d(h->mesh, h->dims[0], h->dims[1], h->dims[2], h->origin_d, h->cell_d, h->grid, h->num_sms, st);
    launch_sdf_slab_min(h->grid, h->dims[0], h->dims[1], h->dims[2], h->slab_min, st);
    h->launches += 2;
    // host verts_f is re-read by the copy above before the next call returns
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return PBF_OK;
}

extern "C" int pbf_sdf_grid_info(pbf_handle* h, int32_t dims[3], double origin[3], double* cell)
{
    if (!h || !dims || !origin || !cell) return set_error(PBF_ERR_INVALID, "null argument");
    if (!h->grid) return set_error(PBF_ERR_STATE, "no SDF grid");
    for (int a = 0; a < 3; ++a) {
        dims[a] = h->dims[a];
        origin[a] = h->mesh_attached ? h->origin_d[a] : (double)h->origin[a];
    }
    *cell = h->mesh_attached ? h->cell_d : (double)h->cell;
    return PBF_OK;
}

extern "C" int pbf_closest_triangle(pbf_handle* h, const float* pts3, uint32_t n, int32_t* out_face, float* out_point3)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    CK(cudaSetDevice(h->device));
    if (!h->mesh_attached) return set_error(PBF_ERR_STATE, "no mesh attached");
    if (n == 0) return PBF_OK;
    if (!pts3 || !out_face || !out_point3) return set_error(PBF_ERR_INVALID, "null argument");
    float *dp = nullptr, *dq = nullptr;
    int* df = nullptr;
    int rc;
    if ((rc = dalloc(dp, 3 * (size_t)n)) || (rc = dalloc(dq, 3 * (size_t)n)) || (rc = dalloc(df, n))) {
        dfree(dp); dfree(dq); dfree(df);
        return rc;
    }
    cudaMemcpyAsync(dp, pts3, 12 * (size_t)n, cudaMemcpyHostToDevice, h->stream);
    launch_mesh_closest(h->mesh, dp, n, df, dq, h->stream);
    ++h->launches;
    cudaMemcpyAsync(out_face, df, 4 * (size_t)n, cudaMemcpyDeviceToHost, h->stream);
    cudaMemcpyAsync(out_point3, dq, 12 * (size_t)n, cudaMemcpyDeviceToHost, h->stream);
    const cudaError_t e = cudaStreamSynchronize(h->stream);
    dfree(dp); dfree(dq); dfree(df);
    if (e != cudaSuccess) return set_error(PBF_ERR_CUDA, "closest_triangle: %s", cudaGetErrorString(e));
    return PBF_OK;
}

extern "C" int pbf_vertex_forces(pbf_handle* h, float band, int use_vel, float* out3, int32_t nv, int32_t* out_contacts)
{
    if (!h) return set_error(PBF_ERR_INVALID, "null handle");
    CK(cudaSetDevice(h->device));
    pbf_handle* o = h->sdf_src;  // the mesh the fluid collides with (possibly borrowed)
    if (!o || !o->mesh_attached) return set_error(PBF_ERR_STATE, "no mesh attached");
    if (nv != o->mesh.nv || !out3) return set_error(PBF_ERR_INVALID, "forces buffer needs %d vertices", o->mesh.nv);
    cudaStream_t st = h->stream;
    if (o != h) CK(cudaStreamSynchronize(o->stream));
    CK(cudaMemsetAsync(o->force_acc, 0, sizeof(long long) * 3 * (size_t)nv, st));
    CK(cudaMemsetAsync(o->force_contacts, 0, sizeof(int), st));
    if (h->contacts_valid && h->n > 0) {
        launch_vertex_forces(o->mesh, h->cand, h->scalars, h->n, band, use_vel, o->force_acc, o->force_contacts, st);
        ++h->launches;
    }
    launch_forces_to_float(nv, o->force_acc, o->force_out, st);
    ++h->launches;
    CK(cudaMemcpyAsync(out3, o->force_out, sizeof(float) * 3 * (size_t)nv, cudaMemcpyDeviceToHost, st));
    int c = 0;
    CK(cudaMemcpyAsync(&c, o->force_contacts, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (out_contacts) *out_contacts = c;
    return PBF_OK;
}
