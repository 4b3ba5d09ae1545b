"""Two-way fluid-solid coupling loop of the reference application
(src/main.cpp:1673-1708 per frame: step, filterContactCandidates,
computeContactForces, deformStep -> syncDeformedMesh), on this engine:

    GPU   fluid step (PBFluids.step)
    GPU   contact candidates + per-vertex forces against the mesh SDF
    host  Laplacian deformation from the forces (pbf_deform_step)
    GPU   LBVH refit + SDF grid recompute of the moved mesh (refitFromMesh)

The reference refreshes the SDF every third deform frame and rebuilds it every
100th (main.cpp:326,335); the GPU refit is cheap enough to run on every frame
the mesh moves, which is what this loop does.
"""
import time

import numpy as np

from . import PBFluids, SDFBoundary, make_particles
from .deform import Deformer, default_params


def c1_deform_params():
    """Scene 1's deformation tuning (include/core/Scene.h:178-188) with its
    lengths scaled from the reference's 3-unit mesh to the 0.4-unit sphere
    (x 0.2/1.5): per-frame clamp 0.00267, total clamp 0.04, contact band 0.016."""
    s = 0.2 / 1.5
    prm = default_params(stiffness=1.0, max_displacement=0.02 * s, max_total_disp=0.30 * s, restore_enabled=1,
                         restore_strength=0.02, control_threshold=1.2, control_threshold_low=1.0)
    return prm, 3, 0.12 * s


class CoupledScene:
    def __init__(self, cfg, pos, vel, verts, faces, anchors, sdf_cell, params, contact_band, kring=3,
                 incremental=True, device=0):
        self.fluid = PBFluids(cfg, device)
        self.fluid.setParticles(make_particles(pos, vel))
        # the step replays one CUDA graph; refitting the mesh SDF rewrites the
        # grid in place, which the graph reads without being re-captured
        self.fluid.set_use_graph(True)
        self.sdf = SDFBoundary(device)
        self.sdf.buildFromMesh(verts, faces, sdf_cell)
        self.fluid.setSDFBoundary(self.sdf)
        self.fluid.setSDFPadding(sdf_cell / 2.0)
        self.fluid.setSDFContainment(False)
        self.deform = Deformer(verts, faces)
        self.deform.set_mode(use_local=not incremental, kring=kring, use_incremental=incremental)
        for a in anchors:
            self.deform.add_anchor(int(a))
        self.params = params
        self.band = float(contact_band)
        self.dt = float(cfg.dt)
        self.rest = np.asarray(verts, np.float64).copy()
        self.times = dict(fluid=0.0, forces=0.0, deform=0.0, refit=0.0)
        self.frames = 0
        self.handles = 0
        self.refactors = 0
        self.contacts = 0

    def frame(self):
        t0 = time.perf_counter()
        self.fluid.step()
        self.fluid.sync()
        t1 = time.perf_counter()
        self.fluid.filterContactCandidates(self.band)
        forces, contacts = self.fluid.computeContactForces(self.band, True)
        t2 = time.perf_counter()
        hc, refactored, moved = self.deform.step(forces, self.dt, self.params)
        t3 = time.perf_counter()
        if moved:
            self.sdf.refitFromMesh(self.deform.vertices())
        t4 = time.perf_counter()
        self.times["fluid"] += t1 - t0
        self.times["forces"] += t2 - t1
        self.times["deform"] += t3 - t2
        self.times["refit"] += t4 - t3
        self.frames += 1
        self.handles = hc
        self.refactors += int(refactored)
        self.contacts = contacts
        return forces, moved
