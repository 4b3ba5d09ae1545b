"""The reference's scene presets and their headless set-up (include/core/
Scene.h, include/core/SceneSetup.h over the C ABI).

    presets()                    the four scenes (pbf_scene_preset structs)
    load_off(path)               (verts (n,3) float64, faces (m,3) int32)
    fit_mesh / place_mesh        fitMeshToDomain / applyMeshTransform
    spawn_particles(cfg)         spawnParticles (PARTICLE_DTYPE records)
    HeadlessScene(index, ...)    a preset loaded into PBFluids + SDFBoundary

The mesh assets are the reference's files (resources/assets/*.off); a caller
points `asset_dir` at its copy of them, or passes `mesh_path` for another
mesh.
"""
import ctypes as C
import os

import numpy as np

from ._capi import FluidConfig, ScenePreset, check, fvec, lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def presets():
    out = []
    for k in range(lib().pbf_scene_count()):
        s = ScenePreset()
        check(lib().pbf_scene_get(k, C.byref(s)))
        out.append(s)
    return out


def load_off(path):
    nv, nf = C.c_int32(), C.c_int32()
    p = os.fsencode(path)
    check(lib().pbf_off_load(p, None, 0, None, 0, C.byref(nv), C.byref(nf)))
    v = np.zeros((nv.value, 3), np.float64)
    f = np.zeros((nf.value, 3), np.int32)
    check(lib().pbf_off_load(p, _ptr(v), nv.value, _ptr(f), nf.value, C.byref(nv), C.byref(nf)))
    return v, f


def fit_center(cfg):
    c = (C.c_float * 3)()
    check(lib().pbf_mesh_fit_center(C.byref(cfg), c))
    return np.array(c[:], np.float32)


def fit_mesh(verts, center, target_size):
    v = np.ascontiguousarray(verts, np.float64).copy()
    check(lib().pbf_mesh_fit(_ptr(v), len(v), fvec(center), float(target_size)))
    return v


def place_mesh(verts, translate, rot_deg):
    v = np.ascontiguousarray(verts, np.float64).copy()
    check(lib().pbf_mesh_place(_ptr(v), len(v), fvec(translate), fvec(rot_deg)))
    return v


def spawn_particles(cfg):
    from . import PARTICLE_DTYPE
    n = C.c_uint32()
    check(lib().pbf_spawn_particles(C.byref(cfg), None, 0, C.byref(n)))
    out = np.zeros(n.value, PARTICLE_DTYPE)
    check(lib().pbf_spawn_particles(C.byref(cfg), _ptr(out), n.value, C.byref(n)))
    return out


def scene_mesh(preset, asset_dir=None, mesh_path=None):
    """The preset's mesh loaded, fitted and placed (loadScene's order)."""
    path = mesh_path or os.path.join(asset_dir or ".", preset.mesh_file.decode())
    v, f = load_off(path)
    v = fit_mesh(v, fit_center(preset.fluid), preset.mesh_fit_size)
    v = place_mesh(v, preset.mesh_translate[:], preset.mesh_rot_deg[:])
    return v, f


class HeadlessScene:
    """A preset applied to a solver and an SDF, as the reference's loadScene +
    confirmAnchorsAndSpawn do (src/main.cpp:959-993, 1192-1243), without a
    window: parameters and walls, the SDF of the placed mesh at the preset's
    cell size, padding and obstacle/container mode, the spawned particles."""

    def __init__(self, index, asset_dir=None, mesh_path=None, device=0):
        from . import PBFluids, SDFBoundary
        self.preset = presets()[index]
        cfg = FluidConfig()
        C.memmove(C.byref(cfg), C.byref(self.preset.fluid), C.sizeof(cfg))
        self.cfg = cfg
        self.verts, self.faces = scene_mesh(self.preset, asset_dir, mesh_path)
        self.fluid = PBFluids(cfg, device=device)
        self.fluid.setBounds(cfg.bounds_min[:], cfg.bounds_max[:], cfg.bound_damping)
        self.sdf = SDFBoundary(device=device)
        self.sdf.buildFromMesh(self.verts, self.faces, self.preset.sdf_cell)
        self.fluid.setSDFBoundary(self.sdf)
        self.fluid.setSDFPadding(self.preset.sdf_padding)
        self.fluid.setSDFContainment(bool(self.preset.sdf_container))
        self.particles = spawn_particles(cfg)
        self.fluid.setParticles(self.particles)

    def step(self):
        self.fluid.step()
