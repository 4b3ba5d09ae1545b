"""Scene presets and headless set-up (include/core/Scene.h,
include/core/SceneSetup.h), host code only.

The presets are compared with the reference's own include/core/Scene.h when
the reference tree is present (this machine); the OFF reader with small
fixtures written here and, when present, the reference's own asset files;
spawnParticles, fitMeshToDomain and the placement with numpy restatements of
src/main.cpp:160-188, 419-432 and 747-770 (lattice and seeded spawns
bit-exact, float32 placement within float32 rounding).
"""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("PBF_REFERENCE_TREE") or os.path.join(os.path.dirname(ROOT), "reference")
F32 = np.float32


def _presets():
    from pbf_b200 import presets
    return presets.presets()


def test_four_presets_with_names_meshes_and_counts():
    ps = _presets()
    assert [p.name.decode() for p in ps] == ["Container Cube", "Surface Cube", "Surface Bull", "Surface Hand"]
    assert [p.mesh_file.decode() for p in ps] == ["cube1538.off", "cube1538.off", "386.off", "200.off"]
    assert [p.sdf_container for p in ps] == [1, 0, 0, 0]
    for p in ps:
        assert p.fluid.particle_count == 1 << 14 and p.fluid.hash_size == 1 << 15
        assert list(p.fluid.bounds_max) == [6.0, 6.0, 6.0] and p.fluid.enable_apbf == 0


def _reference_scene_values(path):
    """Per scene, the numeric `/* label */ value` entries of the reference's
    Scene.h in file order (vectors flattened, strings skipped)."""
    src = open(path).read()
    body = src[src.index("getScenes()"):]
    blocks = re.split(r"\n\s*// \d+ \S+ ", body)[1:]
    out = []
    for b in blocks:
        vals = []
        for m in re.finditer(r"/\*\s*\w[\w ]*?\s*\*/\s*(.*?),[ \t]*(?://[^\n]*)?\n", b):
            raw = m.group(1).strip()
            if raw.startswith('"'):
                continue
            for part in raw.strip("{} ").split(","):
                vals.append(_value(part.strip()))
        out.append(vals)
    return out


def _value(tok):
    tok = tok.replace("f", "").strip() if tok not in ("true", "false") else tok
    if tok == "true":
        return 1.0
    if tok == "false":
        return 0.0
    if "<<" in tok:
        a, b = tok.split("<<")
        return float(int(a) << int(b))
    if "/" in tok:
        a, b = tok.split("/")
        return float(F32(float(a)) / F32(float(b)))
    return float(tok)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "include", "core", "Scene.h")),
                    reason="the reference tree is not on this machine")
def test_presets_equal_reference_scene_header():
    ref = _reference_scene_values(os.path.join(REF, "include", "core", "Scene.h"))
    assert len(ref) == 4
    for p, vals in zip(_presets(), ref):
        f, d = p.fluid, p.deform
        mine = ([f.dt] + list(f.gravity) + [f.h, f.rho0, f.solver_iterations, f.substep_iterations, f.eps,
                                                  f.particle_count] + list(f.spawn_min) + list(f.spawn_max) +
                [f.spawn_random, f.spacing] + list(f.initial_velocity) + list(f.bounds_min) + list(f.bounds_max) +
                [f.bound_damping, f.hash_size, f.enable_scorr, f.k_corr, f.n_corr, f.delta_q, f.cohesion_strength,
                 f.enable_viscosity, f.viscosity, f.interaction_radius, f.interaction_strength, f.enable_vorticity,
                 f.vorticity_epsilon, p.cam_yaw, p.cam_pitch, p.cam_dist, p.point_size, p.mesh_fit_size, p.sdf_cell,
                 p.sdf_padding, p.sdf_container] + list(p.mesh_translate) + list(p.mesh_rot_deg) +
                [d.stiffness, d.max_displacement, d.max_total_disp, d.restore_enabled, d.restore_strength,
                 d.control_threshold, d.control_threshold_low, p.local_kring, p.contact_radius])
        assert len(vals) == len(mine), (len(vals), len(mine))
        np.testing.assert_array_equal(F32(mine), F32(vals))


OFF_FIXTURE = """# a comment before the header\r
\r
NOFF\r
# counts follow\r
5 3 0\r
0 0 0  0 0 1\r
1 0 0  0 0 1\r
# a comment between vertices\r
1 1 0  0 0 1\r
0 1 0 0 0 1\r
0.5 0.5 1 0 0 1\r
4 0 1 2 3\r
3 0 1 4\r
5 0 1 2 3 4\r
"""


def test_off_reader_skips_comments_and_fan_triangulates(tmp_path):
    from pbf_b200 import presets
    p = tmp_path / "fixture.off"
    p.write_bytes(OFF_FIXTURE.encode())
    v, f = presets.load_off(str(p))
    np.testing.assert_array_equal(v, [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0.5, 0.5, 1]])
    # quad -> 2, triangle -> 1, pentagon -> 3 (fans from the first vertex)
    np.testing.assert_array_equal(f, [[0, 1, 2], [0, 2, 3], [0, 1, 4], [0, 1, 2], [0, 2, 3], [0, 3, 4]])
    q = tmp_path / "inline.off"
    q.write_text("OFF 4 1 0\n0 0 0\n1 0 0\n0 1 0\n0 0 1\n3 0 1 2\n")
    v, f = presets.load_off(str(q))
    assert v.shape == (4, 3) and f.tolist() == [[0, 1, 2]]


def test_off_reader_rejects_bad_files(tmp_path):
    from pbf_b200 import presets
    from pbf_b200._capi import PBFError
    bad = tmp_path / "bad.off"
    bad.write_text("PLY\n3 1 0\n")
    short = tmp_path / "short.off"
    short.write_text("OFF\n4 2 0\n0 0 0\n1 0 0\n")
    oob = tmp_path / "oob.off"
    oob.write_text("OFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n3 0 1 3\n")
    huge = tmp_path / "huge.off"
    huge.write_text("OFF\n3 1 0\n0 0 0\n1 0 0\n0 1 0\n2000000000 0 1 2\n")
    for path in (bad, short, oob, huge, tmp_path / "missing.off"):
        with pytest.raises(PBFError):
            presets.load_off(str(path))


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "resources", "assets")),
                    reason="the reference's assets are not on this machine")
@pytest.mark.parametrize("name", ["cube1538.off", "386.off", "200.off"])
def test_reference_assets_load_with_their_declared_counts(name):
    from pbf_b200 import presets
    path = os.path.join(REF, "resources", "assets", name)
    lines = [ln.strip() for ln in open(path) if ln.strip() and not ln.startswith("#")]
    assert "OFF" in lines[0]
    nv, nf = (int(t) for t in lines[1].split()[:2])
    tri = sum(int(ln.split()[0]) - 2 for ln in lines[2 + nv:2 + nv + nf])
    v, f = presets.load_off(path)
    assert v.shape == (nv, 3) and f.shape == (tri, 3)
    assert f.min() >= 0 and f.max() < nv
    np.testing.assert_array_equal(v[0], [float(t) for t in lines[2].split()[:3]])


def lattice_f32(cfg):
    """src/main.cpp:176-184 in float32: z outermost, x innermost."""
    out = []
    step = max(F32(1e-6), F32(cfg.spacing))
    lo = [F32(v) for v in cfg.spawn_min]
    hi = [F32(v) for v in cfg.spawn_max]
    z = lo[2]
    while z <= hi[2] and len(out) < cfg.particle_count:
        y = lo[1]
        while y <= hi[1] and len(out) < cfg.particle_count:
            x = lo[0]
            while x <= hi[0] and len(out) < cfg.particle_count:
                out.append((x, y, z))
                x = F32(x + step)
            y = F32(y + step)
        z = F32(z + step)
    return np.array(out, np.float32).reshape(-1, 3)


def random_f32(cfg):
    """src/main.cpp:164-175: std::mt19937(1337), uniform float in [0, 1) as
    libstdc++ makes it from one 32-bit draw (u / 2^32 in float)."""
    bg = np.random.MT19937()
    bg._legacy_seeding(1337)
    u = bg.random_raw(3 * cfg.particle_count).astype(np.uint32).astype(np.float32) / F32(4294967296.0)
    u = np.where(u >= 1, np.nextafter(F32(1), F32(0)), u).reshape(-1, 3)
    lo = np.array(cfg.spawn_min, np.float32) + F32(cfg.spacing)
    hi = np.array(cfg.spawn_max, np.float32) - F32(cfg.spacing)
    return (lo + (hi - lo) * u).astype(np.float32)


@pytest.mark.parametrize("k", [0, 1, 2, 3])
def test_spawn_lattice_matches_restatement(k):
    from pbf_b200 import presets
    cfg = _presets()[k].fluid
    got = presets.spawn_particles(cfg)
    want = lattice_f32(cfg)
    assert len(got) == len(want) == 1 << 14
    np.testing.assert_array_equal(got["pos"], want)
    np.testing.assert_array_equal(got["pred_pos"], want)
    assert (got["vel"] == 0).all()


def test_spawn_random_matches_restatement():
    from pbf_b200 import presets
    cfg = _presets()[1].fluid
    cfg.spawn_random = 1
    cfg.particle_count = 5000
    cfg.initial_velocity[:] = [0.5, -1.0, 0.25]
    got = presets.spawn_particles(cfg)
    np.testing.assert_array_equal(got["pos"], random_f32(cfg))
    assert np.array_equal(got["vel"], np.tile(F32([0.5, -1.0, 0.25]), (5000, 1)))


def test_fit_and_place_match_restatement():
    from pbf_b200 import presets
    rng = np.random.default_rng(5)
    v = rng.normal(size=(200, 3)) * [3.0, 1.0, 0.5] + [10.0, -2.0, 4.0]
    cfg = _presets()[2].fluid
    c = presets.fit_center(cfg)
    np.testing.assert_array_equal(c, F32([3.0, F32(0.0) + F32(0.4) * F32(6.0), 3.0]))
    got = presets.fit_mesh(v, c, 4.0)
    lo, hi = v.min(0), v.max(0)
    want = (v - 0.5 * (lo + hi)) * (4.0 / (hi - lo).max()) + c.astype(np.float64)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    placed = presets.place_mesh(got, [0.1, 0.2, -0.3], [270.0, 30.0, 90.0])
    lo, hi = got.min(0), got.max(0)
    piv = (F32(0.5) * (lo + hi).astype(np.float32)).astype(np.float32)
    a = np.radians([270.0, 30.0, 90.0])
    Rx = [[1, 0, 0], [0, np.cos(a[0]), -np.sin(a[0])], [0, np.sin(a[0]), np.cos(a[0])]]
    Ry = [[np.cos(a[1]), 0, np.sin(a[1])], [0, 1, 0], [-np.sin(a[1]), 0, np.cos(a[1])]]
    Rz = [[np.cos(a[2]), -np.sin(a[2]), 0], [np.sin(a[2]), np.cos(a[2]), 0], [0, 0, 1]]
    R = np.array(Rx) @ np.array(Ry) @ np.array(Rz)
    want = (got - piv) @ R.T + piv + [0.1, 0.2, -0.3]
    np.testing.assert_allclose(placed, want, rtol=0, atol=5e-6)
