// k_mesh.cu — triangle-mesh SDF on the GPU: LBVH over the faces, refit as
// the mesh deforms, signed-distance grid recompute, closest-triangle queries
// and the per-vertex fluid-to-mesh force reduction.
//
// Replaces the reference's CPU median-split TriangleBVH + OpenMP distance
// grid (src/fluid/SDFBoundary.cpp:78-265,400-465) and the OpenMP contact
// force loop of src/main.cpp:604-710.  The tree is a Karras (2012) radix
// tree over 30-bit Morton codes of the face centroids: internal nodes
// [0, nf-1), leaves [nf-1, 2nf-1), built and refit fully in parallel.  Only
// the node boxes differ from the reference's tree; nearest-point answers are
// the same up to ties between equidistant faces.
#include "pbf_kernels.h"

namespace pbf {

struct Hit {
    float d2;
    float3 p;
    int feature;  // 0 face, 1 AB, 2 AC, 3 BC, 4 A, 5 B, 6 C (SDFBoundary.cpp:17)
    int face;
};

__device__ __forceinline__ float3 f3sub(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float f3dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 f3madd(float3 a, float3 d, float s)
{
    return make_float3(a.x + d.x * s, a.y + d.y * s, a.z + d.z * s);
}

// closestPointOnTriangle (Ericson 5.1.5 with feature, SDFBoundary.cpp:22-54)
__device__ float3 closest_on_triangle(float3 P, float3 A, float3 B, float3 C, int& feature)
{
    const float3 AB = f3sub(B, A), AC = f3sub(C, A), AP = f3sub(P, A);
    const float d1 = f3dot(AB, AP), d2 = f3dot(AC, AP);
    if (d1 <= 0.f && d2 <= 0.f) { feature = 4; return A; }
    const float3 BP = f3sub(P, B);
    const float d3 = f3dot(AB, BP), d4 = f3dot(AC, BP);
    if (d3 >= 0.f && d4 <= d3) { feature = 5; return B; }
    const float3 CP = f3sub(P, C);
    const float d5 = f3dot(AB, CP), d6 = f3dot(AC, CP);
    if (d6 >= 0.f && d5 <= d6) { feature = 6; return C; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) { feature = 1; return f3madd(A, AB, d1 / (d1 - d3)); }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) { feature = 2; return f3madd(A, AC, d2 / (d2 - d6)); }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        feature = 3;
        return f3madd(B, f3sub(C, B), (d4 - d3) / ((d4 - d3) + (d5 - d6)));
    }
    const float denom = 1.0f / (va + vb + vc);
    feature = 0;
    return f3madd(f3madd(A, AB, vb * denom), AC, vc * denom);
}

__device__ __forceinline__ float box_d2(float3 p, float4 lo, float4 hi)
{
    float d2 = 0.f, t;
    if (p.x < lo.x) { t = lo.x - p.x; d2 += t * t; } else if (p.x > hi.x) { t = p.x - hi.x; d2 += t * t; }
    if (p.y < lo.y) { t = lo.y - p.y; d2 += t * t; } else if (p.y > hi.y) { t = p.y - hi.y; d2 += t * t; }
    if (p.z < lo.z) { t = lo.z - p.z; d2 += t * t; } else if (p.z > hi.z) { t = p.z - hi.z; d2 += t * t; }
    return d2;
}

// Branch-and-bound nearest face of the subtree at `root`, nearer child first
// (TriangleBVH::query, SDFBoundary.cpp:225-257, as an explicit stack); the
// first face met with the smallest squared distance wins.
__device__ Hit subtree_closest(const MeshDev& M, float3 P, int root, float bound = 3.0e38f)
{
    Hit best;
    best.d2 = bound;
    best.p = make_float3(0.f, 0.f, 0.f);
    best.feature = 0;
    best.face = -1;
    if (M.nf <= 0 || root < 0) return best;
    const int n_int = M.nf - 1;
    // Depth bound: each internal node splits its range at a strictly longer
    // common prefix of the 64-bit (Morton code, leaf index) keys than its
    // parent did, so no path is longer than 64 internal nodes.  A pop pushes
    // at most two nodes, one of which is popped next, so the stack never holds
    // more than depth + 2 <= 66 entries and kStack is never reached.
    constexpr int kStack = 96;
    int stack[kStack];
    int sp = 0;
    stack[sp++] = root;
    while (sp > 0) {
        const int node = stack[--sp];
        if (box_d2(P, __ldg(M.bmin + node), __ldg(M.bmax + node)) >= best.d2) continue;
        if (node >= n_int) {
            const int f = __ldg(M.leaf_face + (node - n_int));
            const int3 tri = M.faces[f];
            const float3 A = M.verts[tri.x], B = M.verts[tri.y], C = M.verts[tri.z];
            int feat;
            const float3 cp = closest_on_triangle(P, A, B, C, feat);
            const float3 dd = f3sub(P, cp);
            const float d2 = f3dot(dd, dd);
            if (d2 < best.d2) {
                best.d2 = d2;
                best.p = cp;
                best.feature = feat;
                best.face = f;
            }
            continue;
        }
        const int2 ch = __ldg(M.child + node);
        const float dl = box_d2(P, __ldg(M.bmin + ch.x), __ldg(M.bmax + ch.x));
        const float dr = box_d2(P, __ldg(M.bmin + ch.y), __ldg(M.bmax + ch.y));
        // push the farther child first so the nearer one is visited first
        const int nearc = dl <= dr ? ch.x : ch.y, farc = dl <= dr ? ch.y : ch.x;
        const float dnear = fminf(dl, dr), dfar = fmaxf(dl, dr);
        if (dfar < best.d2 && sp < kStack) stack[sp++] = farc;
        if (dnear < best.d2 && sp < kStack) stack[sp++] = nearc;
    }
    return best;
}

__device__ Hit mesh_closest(const MeshDev& M, float3 P) { return subtree_closest(M, P, 0); }

__device__ __forceinline__ float centre_d2(float3 p, float4 lo, float4 hi)
{
    const float x = 0.5f * (lo.x + hi.x) - p.x, y = 0.5f * (lo.y + hi.y) - p.y, z = 0.5f * (lo.z + hi.z) - p.z;
    return x * x + y * y + z * z;
}

// Squared distance to the face reached by taking the nearer child from
// `root` (by box distance, then by box centre when P lies in both boxes, as
// it does inside a closed mesh): an upper bound of the subtree's nearest
// distance.
__device__ float first_leaf_d2(const MeshDev& M, float3 P, int root)
{
    const int n_int = M.nf - 1;
    int node = root;
    while (node < n_int) {
        const int2 ch = __ldg(M.child + node);
        const float4 l0 = __ldg(M.bmin + ch.x), l1 = __ldg(M.bmax + ch.x);
        const float4 r0 = __ldg(M.bmin + ch.y), r1 = __ldg(M.bmax + ch.y);
        const float dl = box_d2(P, l0, l1), dr = box_d2(P, r0, r1);
        const bool left = dl != dr ? dl < dr : centre_d2(P, l0, l1) <= centre_d2(P, r0, r1);
        node = left ? ch.x : ch.y;
    }
    const int f = __ldg(M.leaf_face + (node - n_int));
    const int3 tri = M.faces[f];
    int feat;
    const float3 cp = closest_on_triangle(P, M.verts[tri.x], M.verts[tri.y], M.verts[tri.z], feat);
    const float3 dd = f3sub(P, cp);
    return f3dot(dd, dd);
}

// Position of the subtree at `node` in mesh_closest's visiting order for the
// point P: the near (0) / far (1) choices on the path from the root, root
// first, as the high bits of a key.  Disjoint subtrees compare as their
// first-visited faces do.
__device__ uint32_t visit_rank(const MeshDev& M, float3 P, int node)
{
    uint32_t bits = 0;
    int len = 0;
    for (int c = node, p = M.parent[node]; p >= 0 && len < 32; c = p, p = M.parent[p], ++len) {
        const int2 ch = __ldg(M.child + p);
        const float dl = box_d2(P, __ldg(M.bmin + ch.x), __ldg(M.bmax + ch.x));
        const float dr = box_d2(P, __ldg(M.bmin + ch.y), __ldg(M.bmax + ch.y));
        const int nearc = dl <= dr ? ch.x : ch.y;
        bits |= (c == nearc ? 0u : 1u) << len;
    }
    return len ? bits << (32 - len) : 0u;
}

// ---- LBVH construction ------------------------------------------------------------
__device__ __forceinline__ int delta(const uint32_t* codes, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clz(a ^ b);
}

__global__ void k_lbvh_topology(int n, const uint32_t* __restrict__ codes, int2* __restrict__ child,
                                int* __restrict__ parent)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(codes, n, i, i - d);
    int lmax = 2;
    while (delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(codes, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int n_int = n - 1;
    const int left = (min(i, j) == gamma) ? n_int + gamma : gamma;
    const int right = (max(i, j) == gamma + 1) ? n_int + gamma + 1 : gamma + 1;
    child[i] = make_int2(left, right);
    parent[left] = i;
    parent[right] = i;
    if (i == 0) parent[0] = -1;
}

void launch_lbvh_topology(int nf, const uint32_t* sorted_codes, int2* child, int* parent, cudaStream_t st)
{
    if (nf < 2) return;
    k_lbvh_topology<<<(nf - 1 + 127) / 128, 128, 0, st>>>(nf, sorted_codes, child, parent);
}

__global__ void k_face_normals(int nf, const int3* __restrict__ faces, const float3* __restrict__ verts,
                               float3* __restrict__ fn)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int3 t = faces[f];
    const float3 A = verts[t.x], B = verts[t.y], C = verts[t.z];
    const float3 u = f3sub(B, A), v = f3sub(C, A);
    float3 n = make_float3(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
    const float len = sqrtf(f3dot(n, n));
    if (len > 1e-12f) n = make_float3(n.x / len, n.y / len, n.z / len);  // SDFBoundary.cpp:447-450
    fn[f] = n;
}

// Leaf boxes, then parents once both children are done (arrival counters).
__global__ void k_lbvh_refit(MeshDev M)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= M.nf) return;
    const int n_int = M.nf - 1;
    const int f = M.leaf_face[k];
    const int3 t = M.faces[f];
    const float3 A = M.verts[t.x], B = M.verts[t.y], C = M.verts[t.z];
    int node = n_int + k;
    M.bmin[node] = make_float4(fminf(A.x, fminf(B.x, C.x)), fminf(A.y, fminf(B.y, C.y)), fminf(A.z, fminf(B.z, C.z)), 0.f);
    M.bmax[node] = make_float4(fmaxf(A.x, fmaxf(B.x, C.x)), fmaxf(A.y, fmaxf(B.y, C.y)), fmaxf(A.z, fmaxf(B.z, C.z)), 0.f);
    __threadfence();
    int p = M.parent[node];
    // a Karras tree over 30-bit codes with index tie-breaks is < 64 levels deep;
    // the bound only guards against a malformed topology
    for (int level = 0; p >= 0 && level < 128; ++level) {
        if (atomicAdd(&M.flags[p], 1u) == 0u) return;  // first arrival: the sibling finishes the parent
        const int2 ch = M.child[p];
        const float4 l0 = __ldcg(M.bmin + ch.x), l1 = __ldcg(M.bmax + ch.x);
        const float4 r0 = __ldcg(M.bmin + ch.y), r1 = __ldcg(M.bmax + ch.y);
        M.bmin[p] = make_float4(fminf(l0.x, r0.x), fminf(l0.y, r0.y), fminf(l0.z, r0.z), 0.f);
        M.bmax[p] = make_float4(fmaxf(l1.x, r1.x), fmaxf(l1.y, r1.y), fmaxf(l1.z, r1.z), 0.f);
        __threadfence();
        node = p;
        p = M.parent[node];
    }
}

// ---- pseudo-normals (SDFBoundary.cpp:341-383), from the current face normals --------------
// Angle-weighted vertex normals: each incident face's normal weighted by its
// interior angle at the vertex, summed in ascending face order (the order of
// the reference's loop over faces), then normalised if longer than 1e-12.
// vfc[voff[v] .. voff[v+1]) lists (face, corner) of vertex v by face.
__global__ void k_vertex_normals(int nv, const int3* __restrict__ faces, const float3* __restrict__ verts,
                                 const float3* __restrict__ fn, const int* __restrict__ voff,
                                 const int2* __restrict__ vfc, float3* __restrict__ vn)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    float3 s = make_float3(0.f, 0.f, 0.f);
    for (int k = voff[v]; k < voff[v + 1]; ++k) {
        const int2 e = vfc[k];
        const int3 t = faces[e.x];
        const int idx[3] = {t.x, t.y, t.z};
        const float3 p = verts[idx[e.y]];
        float3 a = f3sub(verts[idx[e.y == 0 ? 1 : 0]], p), b = f3sub(verts[idx[e.y == 2 ? 1 : 2]], p);
        const float la = sqrtf(f3dot(a, a)), lb = sqrtf(f3dot(b, b));
        if (la > 0.f) a = make_float3(a.x / la, a.y / la, a.z / la);
        if (lb > 0.f) b = make_float3(b.x / lb, b.y / lb, b.z / lb);
        const float ang = acosf(fminf(1.f, fmaxf(-1.f, f3dot(a, b))));
        const float3 n = fn[e.x];
        s = make_float3(s.x + ang * n.x, s.y + ang * n.y, s.z + ang * n.z);
    }
    const float len = sqrtf(f3dot(s, s));
    if (len > 1e-12f) s = make_float3(s.x / len, s.y / len, s.z / len);
    vn[v] = s;
}

// Edge normals: for slot 3f + k (edges AB, AC, BC of face f), the normalised
// sum of the two face normals of an edge shared by exactly two faces
// (partner = the other face, -1 otherwise); the face normal when there is
// no partner or the sum is shorter than 1e-12 (a 180-degree fold).
__global__ void k_edge_normals(int nf, const float3* __restrict__ fn, const int* __restrict__ partner,
                               float3* __restrict__ en)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * nf) return;
    const int f = i / 3, q = partner[i];
    float3 n = fn[f];
    if (q >= 0) {
        const float3 o = fn[q];
        const float3 sm = make_float3(n.x + o.x, n.y + o.y, n.z + o.z);
        const float len = sqrtf(f3dot(sm, sm));
        if (len >= 1e-12f) n = make_float3(sm.x / len, sm.y / len, sm.z / len);
    }
    en[i] = n;
}

void launch_mesh_pseudo_normals(MeshDev M, const int* voff, const int2* vfc, const int* partner, float3* vert_n,
                                float3* edge_n, cudaStream_t st, uint64_t* launches)
{
    if (M.nf <= 0) return;
    k_vertex_normals<<<(M.nv + 127) / 128, 128, 0, st>>>(M.nv, M.faces, M.verts, M.face_n, voff, vfc, vert_n);
    k_edge_normals<<<(3 * M.nf + 127) / 128, 128, 0, st>>>(M.nf, M.face_n, partner, edge_n);
    if (launches) *launches += 2;
}

void launch_mesh_refit(MeshDev M, cudaStream_t st, uint64_t* launches)
{
    if (M.nf <= 0) return;
    k_face_normals<<<(M.nf + 127) / 128, 128, 0, st>>>(M.nf, M.faces, M.verts, M.face_n);
    if (M.nf > 1) cudaMemsetAsync(M.flags, 0, sizeof(uint32_t) * (size_t)(M.nf - 1), st);
    k_lbvh_refit<<<(M.nf + 127) / 128, 128, 0, st>>>(M);
    if (launches) *launches += 2;
}

// ---- signed distance grid (SDFBoundary::recomputeDistances + signedDistanceAt)
__device__ __forceinline__ float3 pseudo_normal(const MeshDev& M, const Hit& h)
{
    switch (h.feature) {
    case 0: return M.face_n[h.face];
    case 1: return M.edge_n[3 * h.face + 0];
    case 2: return M.edge_n[3 * h.face + 1];
    case 3: return M.edge_n[3 * h.face + 2];
    default: {
        const int3 t = M.faces[h.face];
        const int v = h.feature == 4 ? t.x : (h.feature == 5 ? t.y : t.z);
        return M.vert_n[v];
    }
    }
}

// One warp per voxel: lane l searches the subtree at M.frontier[l] (the
// frontier covers the tree) for faces within the warp's bound U, then the
// warp keeps the smallest squared distance and, among equal ones, the
// subtree mesh_closest would visit first.  Within a subtree the search is mesh_closest's, so the winner is the
// face, point and feature a single mesh_closest walk returns; the walk's
// length is split over 32 lanes (a voxel deep inside a closed mesh has almost
// every face within its bound).
__global__ void __launch_bounds__(128) k_mesh_grid(MeshDev M, int dx, int dy, int dz, double ox, double oy,
                                                   double oz, double cell, float* __restrict__ out)
{
    const long total = (long)dx * dy * dz;
    const int lane = threadIdx.x & 31;
    const long warps = (long)gridDim.x * (blockDim.x >> 5);
    const int root = M.frontier[lane];
    for (long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < total; i += warps) {
        const int z = (int)(i % dz);
        const int y = (int)((i / dz) % dy);
        const int x = (int)(i / ((long)dy * dz));
        const float3 P = make_float3((float)(ox + x * cell), (float)(oy + y * cell), (float)(oz + z * cell));
        // U: the smallest first-leaf distance over the lanes, reached by some
        // face, so the nearest distance is <= U; a lane then searches only for
        // faces within U (the bound just above U keeps faces at exactly U)
        const uint32_t ub = __reduce_min_sync(0xFFFFFFFFu,
                                              root >= 0 ? __float_as_uint(first_leaf_d2(M, P, root)) : 0x7F7FFFFFu);
        const Hit h = subtree_closest(M, P, root, nextafterf(__uint_as_float(ub), 3.0e38f));
        const uint32_t d2b = __float_as_uint(h.d2);  // non-negative: bit order = value order
        const uint32_t rank = root >= 0 ? visit_rank(M, P, root) : 0xFFFFFFFFu;
        const uint32_t dmin = __reduce_min_sync(0xFFFFFFFFu, d2b);
        const uint32_t rmin = __reduce_min_sync(0xFFFFFFFFu, d2b == dmin ? rank : 0xFFFFFFFFu);
        const uint32_t win = __ballot_sync(0xFFFFFFFFu, d2b == dmin && rank == rmin);
        if (lane == __ffs(win) - 1) {
            float d = 0.0f;
            if (h.face >= 0) {
                const float3 pn = pseudo_normal(M, h);
                const float s = (f3dot(f3sub(P, h.p), pn) >= 0.0f) ? 1.0f : -1.0f;
                d = s * sqrtf(h.d2);
            }
            out[i] = d;
        }
    }
}

void launch_mesh_grid_d(MeshDev M, int dx, int dy, int dz, const double* o, double cell, float* out, int sms,
                        cudaStream_t st)
{
    const long total = (long)dx * dy * dz;
    long blocks = (total + 3) / 4;  // four voxels (warps) per block
    if (blocks > (long)sms * 16) blocks = (long)sms * 16;
    if (blocks < 1) blocks = 1;
    k_mesh_grid<<<(unsigned)blocks, 128, 0, st>>>(M, dx, dy, dz, o[0], o[1], o[2], cell, out);
}

__global__ void k_mesh_closest(MeshDev M, const float* __restrict__ pts, uint32_t n, int* __restrict__ face,
                               float* __restrict__ point)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Hit h = mesh_closest(M, make_float3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]));
    face[i] = h.face;
    point[3 * i] = h.p.x;
    point[3 * i + 1] = h.p.y;
    point[3 * i + 2] = h.p.z;
}

void launch_mesh_closest(MeshDev M, const float* pts3, uint32_t n, int* face, float* point3, cudaStream_t st)
{
    if (n == 0) return;
    k_mesh_closest<<<(n + 127) / 128, 128, 0, st>>>(M, pts3, n, face, point3);
}

// ---- per-vertex contact forces (computeContactForces, src/main.cpp:604-710) ----
// barycentric (src/main.cpp:557-571) in double, clamped and renormalised.
__device__ void barycentric_d(float3 Pt, float3 A, float3 B, float3 C, double& u, double& v, double& w)
{
    const double v0x = (double)B.x - A.x, v0y = (double)B.y - A.y, v0z = (double)B.z - A.z;
    const double v1x = (double)C.x - A.x, v1y = (double)C.y - A.y, v1z = (double)C.z - A.z;
    const double v2x = (double)Pt.x - A.x, v2y = (double)Pt.y - A.y, v2z = (double)Pt.z - A.z;
    const double d00 = v0x * v0x + v0y * v0y + v0z * v0z;
    const double d01 = v0x * v1x + v0y * v1y + v0z * v1z;
    const double d11 = v1x * v1x + v1y * v1y + v1z * v1z;
    const double d20 = v2x * v0x + v2y * v0y + v2z * v0z;
    const double d21 = v2x * v1x + v2y * v1y + v2z * v1z;
    const double denom = d00 * d11 - d01 * d01;
    if (fabs(denom) < 1e-20) { u = 1.0; v = 0.0; w = 0.0; return; }
    const double vv = (d11 * d20 - d01 * d21) / denom;
    const double ww = (d00 * d21 - d01 * d20) / denom;
    double uu = fmax(0.0, 1.0 - vv - ww), vc = fmax(0.0, vv), wc = fmax(0.0, ww);
    const double s = uu + vc + wc;
    if (s > 1e-20) { uu /= s; vc /= s; wc /= s; }
    u = uu; v = vc; w = wc;
}

constexpr double kFixScale = 4294967296.0;  // 2^32

__global__ void k_vertex_forces(MeshDev M, const float4* __restrict__ cand, const uint32_t* __restrict__ count,
                                uint32_t cap, float band, int use_vel, long long* __restrict__ acc,
                                int* __restrict__ contacts)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t cnt = min(*count, cap);
    if (c >= cnt) return;
    const float4 p4 = cand[2 * c], v4 = cand[2 * c + 1];
    const float3 P = make_float3(p4.x, p4.y, p4.z);
    const Hit h = mesh_closest(M, P);
    if (h.face < 0) return;
    const float3 to = f3sub(h.p, P);
    const float dist = sqrtf(f3dot(to, to));
    if (dist > band) return;  // :642
    float3 dir;
    if (dist > 1e-6f) {
        dir = make_float3(to.x / dist, to.y / dist, to.z / dist);
    } else {
        const float3 n = M.face_n[h.face];  // (B-A)x(C-A) normalised, outward
        dir = make_float3(-n.x, -n.y, -n.z);
    }
    float mag = 1.0f;
    if (use_vel) {
        mag = fmaxf(0.0f, v4.x * dir.x + v4.y * dir.y + v4.z * dir.z);
        if (mag <= 0.0f) return;
    }
    const int3 t = M.faces[h.face];
    double u, v, w;
    barycentric_d(h.p, M.verts[t.x], M.verts[t.y], M.verts[t.z], u, v, w);
    const double F[3] = {(double)dir.x * mag, (double)dir.y * mag, (double)dir.z * mag};
    const int vi[3] = {t.x, t.y, t.z};
    const double wt[3] = {u, v, w};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const long long q = __double2ll_rn(F[a] * wt[k] * kFixScale);
            if (q) atomicAdd((unsigned long long*)&acc[3 * vi[k] + a], (unsigned long long)q);
        }
    atomicAdd(contacts, 1);
}

void launch_vertex_forces(MeshDev M, const float4* cand, const uint32_t* count, uint32_t cap, float band,
                          int use_vel, long long* acc3, int* contacts, cudaStream_t st)
{
    if (cap == 0) return;
    k_vertex_forces<<<(cap + 127) / 128, 128, 0, st>>>(M, cand, count, cap, band, use_vel, acc3, contacts);
}

__global__ void k_forces_to_float(int nv, const long long* __restrict__ acc, float* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 3 * nv) out[i] = (float)((double)acc[i] / kFixScale);
}

void launch_forces_to_float(int nv, const long long* acc3, float* out3, cudaStream_t st)
{
    if (nv <= 0) return;
    k_forces_to_float<<<(3 * nv + 255) / 256, 256, 0, st>>>(nv, acc3, out3);
}

// ---- Morton codes of face centroids -------------------------------------------------------
__device__ __forceinline__ uint32_t expand_bits(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_morton(int nf, const int3* __restrict__ faces, const float3* __restrict__ verts, float3 lo,
                         float3 inv_ext, uint32_t* __restrict__ codes)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int3 t = faces[f];
    const float3 A = verts[t.x], B = verts[t.y], C = verts[t.z];
    const float cx = (A.x + B.x + C.x) * (1.0f / 3.0f), cy = (A.y + B.y + C.y) * (1.0f / 3.0f),
                cz = (A.z + B.z + C.z) * (1.0f / 3.0f);
    const float ux = fminf(fmaxf((cx - lo.x) * inv_ext.x, 0.f), 1.f);
    const float uy = fminf(fmaxf((cy - lo.y) * inv_ext.y, 0.f), 1.f);
    const float uz = fminf(fmaxf((cz - lo.z) * inv_ext.z, 0.f), 1.f);
    const uint32_t ix = min((uint32_t)(ux * 1024.f), 1023u), iy = min((uint32_t)(uy * 1024.f), 1023u),
                   iz = min((uint32_t)(uz * 1024.f), 1023u);
    codes[f] = (expand_bits(ix) << 2) | (expand_bits(iy) << 1) | expand_bits(iz);
}

void launch_morton(int nf, const int3* faces, const float3* verts, float3 lo, float3 inv_ext, uint32_t* codes,
                   cudaStream_t st)
{
    if (nf <= 0) return;
    k_morton<<<(nf + 127) / 128, 128, 0, st>>>(nf, faces, verts, lo, inv_ext, codes);
}

}  // namespace pbf
