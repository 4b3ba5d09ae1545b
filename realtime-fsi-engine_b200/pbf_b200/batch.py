"""Helpers around the multi-scene engine: building a batch from generated
scenes, the one-handle-per-scene sequential form it is compared with, and
the partition of scenes across ranks (scenes are independent, so a multi-GPU
run shards them with no per-step exchange)."""
import ctypes as C

import numpy as np

from . import Batch, GridSDF, PBFluids, make_particles
from ._capi import FluidConfig


def scene_config(cfg, scene):
    """The single-scene FluidConfig equivalent to one scene of a batch."""
    c = FluidConfig()
    C.memmove(C.byref(c), C.byref(cfg), C.sizeof(c))
    c.bounds_min[:] = list(scene["bounds_min"])
    c.bounds_max[:] = list(scene["bounds_max"])
    c.hash_size = int(scene.get("hash_size", 0)) or cfg.hash_size
    c.particle_count = int(scene["n"])
    return c


def make_batch(cfg, scenes, device=0):
    """Batch holding `scenes` (dicts of scenes.c3) with particles and SDFs set."""
    b = Batch(cfg, scenes, device)
    for k, s in enumerate(scenes):
        b.set_particles(k, make_particles(s["pos"], s["vel"]))
        if s.get("sdf") is not None:
            grid, origin, cell, pad = s["sdf"]
            b.set_sdf_grid(k, grid, origin, cell)
            b.set_sdf_mode(k, pad, False)
    return b


def make_sequential(cfg, scenes, device=0):
    """One PBFluids per scene with the same configuration (the sequential
    form of the batch); returns [(fluid, sdf)] (the SDF objects must stay
    alive with their fluids)."""
    out = []
    for s in scenes:
        f = PBFluids(scene_config(cfg, s), device)
        f.setParticles(make_particles(s["pos"], s["vel"]))
        sdf = None
        if s.get("sdf") is not None:
            grid, origin, cell, pad = s["sdf"]
            sdf = GridSDF(grid, origin, cell, device)
            f.setSDFBoundary(sdf)
            f.setSDFPadding(pad)
        out.append((f, sdf))
    return out


def partition_scenes(sizes, world_size):
    """Greedy balance of scene sizes over ranks: scenes in decreasing size,
    each to the currently lightest rank (ties to the lower rank).  Returns a
    list of scene-index lists, each in increasing index order."""
    sizes = np.asarray(sizes, dtype=np.int64)
    load = [0] * world_size
    parts = [[] for _ in range(world_size)]
    for k in sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i)):
        r = min(range(world_size), key=lambda j: (load[j], j))
        parts[r].append(k)
        load[r] += int(sizes[k])
    return [sorted(p) for p in parts]
