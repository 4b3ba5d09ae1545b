"""The reference's four scene presets (include/core/Scene.h) set up headless
(include/core/SceneSetup.h: OFF mesh -> fit -> placement -> SDF -> spawn) and
stepped 100 frames on the GPU.

The reference's asset files are not available where the GPU tests run, so
each preset's mesh is replaced by a stand-in written here as an OFF file and
read back through the OFF reader: the cube assets by a cube of the same
topology (a 16 x 16 grid per face: 1,538 vertices, 3,072 triangles), the bull
and the hand by closed ellipsoids of similar proportions.  Checked after 100
frames: the preset's particle count, finite state, every particle inside the
walls, the container scene's fluid still inside its cube, and the obstacle
scenes' fluid outside their meshes.
"""
import math

import numpy as np
import pytest


def grid_cube(n=16):
    """Cube [-0.5, 0.5]^3 with an n x n grid of quads per face, triangles
    wound outward; shared edge and corner vertices merged."""
    index = {}
    verts = []

    def vid(p):
        key = tuple(int(round(c * 2 * n)) for c in p)
        if key not in index:
            index[key] = len(verts)
            verts.append(p)
        return index[key]

    faces = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            u, v = (axis + 1) % 3, (axis + 2) % 3
            for i in range(n):
                for j in range(n):
                    quad = []
                    for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        p = [0.0, 0.0, 0.0]
                        p[axis] = 0.5 * sign
                        p[u] = -0.5 + (i + di) / n
                        p[v] = -0.5 + (j + dj) / n
                        quad.append(vid(tuple(p)))
                    a, b, c, d = quad
                    # (u, v, axis) is right-handed: counter-clockwise seen from +axis
                    if sign > 0:
                        faces += [(a, b, c), (a, c, d)]
                    else:
                        faces += [(a, c, b), (a, d, c)]
    return np.array(verts), np.array(faces, np.int32)


def ellipsoid(radii, n_lat=24, n_lon=48):
    verts = [(0.0, 0.0, radii[2])]
    for i in range(1, n_lat):
        th = math.pi * i / n_lat
        for j in range(n_lon):
            ph = 2 * math.pi * j / n_lon
            verts.append((radii[0] * math.sin(th) * math.cos(ph), radii[1] * math.sin(th) * math.sin(ph),
                          radii[2] * math.cos(th)))
    verts.append((0.0, 0.0, -radii[2]))
    last = len(verts) - 1
    faces = []
    for j in range(n_lon):
        faces.append((0, 1 + j, 1 + (j + 1) % n_lon))
    for i in range(n_lat - 2):
        r0, r1 = 1 + i * n_lon, 1 + (i + 1) * n_lon
        for j in range(n_lon):
            a, b = r0 + j, r0 + (j + 1) % n_lon
            c, d = r1 + j, r1 + (j + 1) % n_lon
            faces += [(a, c, d), (a, d, b)]
    r0 = 1 + (n_lat - 2) * n_lon
    for j in range(n_lon):
        faces.append((last, r0 + (j + 1) % n_lon, r0 + j))
    return np.array(verts), np.array(faces, np.int32)


def write_off(path, v, f):
    with open(path, "w") as fh:
        fh.write("OFF\n# stand-in mesh\n%d %d 0\n" % (len(v), len(f)))
        for p in v:
            fh.write("%.9g %.9g %.9g\n" % tuple(p))
        for t in f:
            fh.write("3 %d %d %d\n" % tuple(t))


STAND_INS = {"cube1538.off": lambda: grid_cube(16), "386.off": lambda: ellipsoid((1.0, 0.45, 0.6)),
             "200.off": lambda: ellipsoid((0.45, 1.0, 0.15))}


def test_stand_in_cube_has_the_asset_topology():
    v, f = grid_cube(16)
    assert len(v) == 1538 and len(f) == 3072
    # closed and outward: the divergence theorem gives the volume, positive
    a, b, c = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    assert abs(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0 - 1.0) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_preset_steps_100_frames_headless(have_gpu, tmp_path, k):
    from pbf_b200 import presets
    pre = presets.presets()[k]
    name = pre.mesh_file.decode()
    v, f = STAND_INS[name]()
    path = tmp_path / name
    write_off(str(path), v, f)
    sc = presets.HeadlessScene(k, mesh_path=str(path))
    n = len(sc.particles)
    assert n == pre.fluid.particle_count == 1 << 14
    x0 = sc.particles["pos"].astype(np.float64)
    for _ in range(100):
        sc.step()
    out = sc.fluid.readbackParticles()
    x = out["pos"].astype(np.float64)
    assert np.isfinite(x).all() and np.isfinite(out["vel"]).all()
    lo, hi = np.array(pre.fluid.bounds_min[:]), np.array(pre.fluid.bounds_max[:])
    assert (x >= lo - 1e-6).all() and (x <= hi + 1e-6).all()
    d = sc.sdf.sample(x)
    cell = pre.sdf_cell
    if pre.sdf_container:
        assert (d < 0).mean() >= 0.99, (d >= 0).sum()
    else:
        assert (d < -cell).mean() <= 0.005, (d < -cell).sum()
    # the fluid fell or spread: it moved
    assert np.abs(x - x0).max() > 0.1
