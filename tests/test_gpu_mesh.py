"""Triangle-mesh SDF on the GPU (LBVH build/refit/rebuild, pseudo-normals,
grid, closest triangle, per-vertex contact forces) against the FP64
restatement of src/fluid/SDFBoundary.cpp and src/main.cpp:604-710, and
directly against the reference's own SDFBoundary (fixture sdf_ref.npz, made
by compiling SDFBoundary.cpp here; the restatement equals it bit for bit,
tests/test_oracle_golden.py).  The GPU computes in FP32: grids agree within
2e-6, the analytic sphere bounds both.
"""
import os

import ctypes as C

import numpy as np
import pytest

import oracle as O
import pbf_b200 as P
import pbfh as H
from pbf_b200 import scenes

pytestmark = pytest.mark.gpu


def oracle_mesh(V, F, cell):
    V = np.ascontiguousarray(V, np.float64)
    F = np.ascontiguousarray(F, np.int32)
    m = O.lib().orc_mesh_build(V.reshape(-1), len(V), F.reshape(-1), len(F), float(cell))
    dims = np.zeros(3, np.int32)
    org = np.zeros(3)
    c = C.c_double()
    O.lib().orc_mesh_grid_info(m, dims, org, C.byref(c))
    return m, dims, org


def oracle_grid(m, dims):
    out = np.zeros(int(np.prod(dims)), np.float32)
    O.lib().orc_mesh_grid(m, out)
    return out


@pytest.mark.parametrize("subdiv,cell", [(1, 0.05), (3, 0.02), (4, 0.0125)])
def test_mesh_grid_matches_oracle(have_gpu, subdiv, cell):
    V, F = scenes.icosphere(subdiv, 0.2, (0.8, 0.3, 0.5))
    sdf = P.SDFBoundary()
    sdf.buildFromMesh(V, F, cell)
    m, dims, org = oracle_mesh(V, F, cell)
    try:
        assert np.array_equal(sdf.dimensions(), dims)
        assert np.allclose(sdf.origin(), org, rtol=0, atol=1e-12)
        g = sdf.distances()
        o = oracle_grid(m, dims)
        assert np.abs(g - o).max() < 2e-6
        # the signed field is a sphere up to the faceting error
        idx = np.indices(dims).reshape(3, -1).T
        P_ = org + idx * cell
        exact = np.linalg.norm(P_ - np.array([0.8, 0.3, 0.5]), axis=1) - 0.2
        assert np.abs(o - exact).max() < 0.2 * (1 - np.cos(np.pi / (5 * 2 ** subdiv))) * 4 + 1e-3
    finally:
        O.lib().orc_mesh_free(m)


def test_refit_after_deformation_matches_oracle(have_gpu):
    V, F = scenes.icosphere(3, 0.2, (0.8, 0.3, 0.5))
    cell = 0.02
    sdf = P.SDFBoundary()
    sdf.buildFromMesh(V, F, cell)
    m, dims, _ = oracle_mesh(V, F, cell)
    try:
        rng = np.random.default_rng(4)
        V2 = V + rng.normal(0, 0.004, V.shape)
        V2[:, 1] -= 0.03 * (V2[:, 1] > 0.4)  # a dent on top
        sdf.refitFromMesh(V2)
        O.lib().orc_mesh_refit(m, np.ascontiguousarray(V2).reshape(-1))
        assert np.abs(sdf.distances() - oracle_grid(m, dims)).max() < 2e-6
        # refitDirty reports movement beyond moveEps only
        assert sdf.refitDirty(V2 + 1e-6, 0.05, 1e-4) is False
        assert sdf.refitDirty(V2 + 1e-3, 0.05, 1e-4) is True
    finally:
        O.lib().orc_mesh_free(m)


def test_build_refit_rebuild_match_reference_sdfboundary(have_gpu):
    """The reference's own SDFBoundary on an icosphere: the GPU grid after a
    build, after refitFromMesh of moved vertices (build-time edge and vertex
    pseudo-normals kept) and after buildFromMesh of the moved vertices (all
    pseudo-normals recomputed on the GPU: pbf_rebuild_mesh), and the closest
    points at seeded queries."""
    z = H.load("sdf_ref.npz")
    cell = float(z["cell"])
    sdf = P.SDFBoundary()
    sdf.buildFromMesh(z["verts"], z["faces"], cell)
    assert np.array_equal(sdf.dimensions(), z["dims"])
    assert np.allclose(sdf.origin(), z["origin"], rtol=0, atol=1e-12)
    assert np.abs(sdf.distances() - z["grid"]).max() < 2e-6
    _, point = sdf.closest_many(z["query"])
    assert np.abs(point - z["closest_point"]).max() < 2e-6
    sdf.refitFromMesh(z["verts_moved"])
    assert np.abs(sdf.distances() - z["refit_grid"]).max() < 2e-6
    sdf.buildFromMesh(z["verts_moved"], z["faces"], cell)  # same faces: the GPU rebuild
    assert np.array_equal(sdf.dimensions(), z["rebuild_dims"])
    assert np.allclose(sdf.origin(), z["rebuild_origin"], rtol=0, atol=1e-12)
    assert np.abs(sdf.distances() - z["rebuild_grid"]).max() < 2e-6


def test_gpu_rebuild_equals_fresh_build(have_gpu):
    """pbf_rebuild_mesh (moved vertices, cached face adjacency) gives the grid
    a fresh pbf_set_sdf_mesh of the moved mesh gives, bit for bit, including
    new grid dimensions when the bounding box grows."""
    V, F = scenes.icosphere(4, 0.2, (0.8, 0.3, 0.5))
    rng = np.random.default_rng(9)
    V2 = V + rng.normal(0, 0.003, V.shape)
    V2[V2[:, 1] > 0.45] += [0.0, 0.05, 0.0]  # the top pulled up: a taller box
    a = P.SDFBoundary()
    a.buildFromMesh(V, F, 0.0125)
    d0 = a.dimensions()
    a.buildFromMesh(V2, F, 0.0125)
    b = P.SDFBoundary()
    b.buildFromMesh(V2, F, 0.0125)
    assert not np.array_equal(a.dimensions(), d0)
    assert np.array_equal(a.dimensions(), b.dimensions())
    assert np.array_equal(a.distances(), b.distances())
    m, dims, _ = oracle_mesh(V2, F, 0.0125)
    try:
        assert np.abs(a.distances() - oracle_grid(m, dims)).max() < 2e-6
    finally:
        O.lib().orc_mesh_free(m)


def test_grid_is_the_single_walk_distance(have_gpu):
    """The grid kernel splits each voxel's nearest-face search over 32 subtrees
    of the LBVH; every voxel's |distance| is the one the single-walk
    closest-triangle query finds at the voxel centre, before and after a
    refit of a deformed mesh (no longer symmetric)."""
    for subdiv, cell in [(1, 0.05), (4, 0.0125)]:
        V, F = scenes.icosphere(subdiv, 0.2, (0.8, 0.3, 0.5))
        sdf = P.SDFBoundary()
        sdf.buildFromMesh(V, F, cell)
        rng = np.random.default_rng(subdiv)
        for verts in (None, V + rng.normal(0, 0.003, V.shape)):
            if verts is not None:
                sdf.refitFromMesh(verts)
            dims, org = sdf.dimensions(), sdf.origin()
            idx = np.indices(dims).reshape(3, -1).T
            pts = (org + idx * cell).astype(np.float32)
            _, point = sdf.closest_many(pts)
            walk = np.sqrt(((point.astype(np.float64) - pts) ** 2).sum(1))
            g = sdf.distances()
            assert np.abs(np.abs(g) - walk).max() < 2e-7
            assert (g < 0).sum() > 0 and (g > 0).sum() > 0


def test_closest_triangle_matches_oracle(have_gpu):
    V, F = scenes.icosphere(3, 0.2, (0.8, 0.3, 0.5))
    sdf = P.SDFBoundary()
    sdf.buildFromMesh(V, F, 0.02)
    m, _, _ = oracle_mesh(V, F, 0.02)
    try:
        pts = np.random.default_rng(6).uniform(0.4, 1.2, size=(3000, 3)).astype(np.float32)
        faces, points = sdf.closest_many(pts)
        for i in range(len(pts)):
            q = np.zeros(3)
            d2 = C.c_double()
            f = O.lib().orc_mesh_closest(m, np.ascontiguousarray(pts[i], np.float64), q, C.byref(d2))
            dg = np.linalg.norm(points[i] - pts[i])
            # the same nearest distance; on a near-tie (two faces equally near
            # within FP32 rounding) either face is a valid answer
            assert abs(dg - np.sqrt(d2.value)) < 2e-6
            if f != faces[i]:
                assert np.linalg.norm(points[i] - q) < 5e-4
    finally:
        O.lib().orc_mesh_free(m)


def test_vertex_forces_match_oracle(have_gpu):
    V, F = scenes.icosphere(3, 0.2, (0.5, 0.3, 0.5))
    cfg, pos, vel = scenes.c0(28, seed=2)
    # a block of fluid (0.56 wide) around the sphere, moving toward it
    pos = (pos - pos.mean(0) + np.array([0.5, 0.3, 0.5])).astype(np.float32)
    pos = pos[np.linalg.norm(pos - np.array([0.5, 0.3, 0.5]), axis=1) > 0.21]
    vel = (np.array([0.5, 0.3, 0.5]) - pos).astype(np.float32)
    cfg.particle_count = len(pos)
    sdf = P.SDFBoundary()
    sdf.buildFromMesh(V, F, 0.02)
    fl = P.PBFluids(cfg)
    fl.setParticles(P.make_particles(pos, vel))
    fl.setSDFBoundary(sdf)
    fl.setSDFPadding(0.01)
    band = 0.06
    fl.filterContactCandidates(band)
    cand = fl.readbackContactCandidates()
    assert len(cand) > 50
    forces, contacts = fl.computeContactForces(band, True)
    m, _, _ = oracle_mesh(V, F, 0.02)
    try:
        ref = np.zeros(3 * len(V))
        cc = np.ascontiguousarray(cand)
        oc = O.lib().orc_contact_forces(m, cc.ctypes.data_as(C.c_void_p), len(cc), band, 1, ref)
        ref = ref.reshape(-1, 3)
        assert contacts == oc > 0
        # per vertex: a candidate whose nearest point sits on a shared edge can
        # split its push over the two faces' corners differently in FP32 and
        # FP64 (near-ties); the barycentric weights of each candidate sum to
        # one, so the total push is conserved tightly
        scale = max(np.abs(ref).max(), 1.0)
        assert np.abs(forces - ref).max() < 1e-3 * scale
        assert np.abs(forces.sum(0) - ref.sum(0)).max() < 1e-5 * max(np.abs(ref.sum(0)).max(), 1.0) * len(cand)
        # deterministic: a second reduction gives the same bits
        f2, _ = fl.computeContactForces(band, True)
        assert np.array_equal(forces, f2)
    finally:
        O.lib().orc_mesh_free(m)


def test_fluid_collides_with_mesh_sdf(have_gpu):
    V, F = scenes.icosphere(3, 0.2, (0.8, 0.3, 0.5))
    cfg, pos, vel = scenes.c0(12, seed=3)
    pos = (pos + np.array([0.68, 0.55, 0.38])).astype(np.float32)
    cfg.enable_scorr = 0
    sdf = P.SDFBoundary()
    sdf.buildFromMesh(V, F, 0.02)
    fl = P.PBFluids(cfg)
    fl.setParticles(P.make_particles(pos, vel))
    fl.setSDFBoundary(sdf)
    fl.setSDFPadding(0.01)
    for _ in range(30):
        fl.step()
    out = fl.readbackParticles()
    r = np.linalg.norm(out["pos"] - np.array([0.8, 0.3, 0.5]), axis=1)
    assert r.min() > 0.2 - 0.01  # nobody tunnels into the sphere
    assert fl.check_finite() == 0
