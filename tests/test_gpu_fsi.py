"""Two-way coupling loop (pbf_b200.fsi): GPU fluid, GPU vertex forces, host
deformation, GPU SDF refit, frame after frame.

Checks: the fluid pushes the sphere (contacts and forces appear, handles
form, vertices move inward within the per-frame and total clamps); the SDF
the fluid collides with tracks the deformed mesh (its grid equals a fresh
build from the deformed vertices); anchors stay put; no non-finite state.
"""
import numpy as np
import pytest

import pbf_b200 as P
from pbf_b200 import fsi, scenes

pytestmark = pytest.mark.gpu


def small_c1():
    cfg, pos, vel, V, F, anchors = scenes.c1()
    # a 24^3 block of the C1 lattice right above a subdivision-3 sphere
    d = 0.0125
    pos = scenes.lattice(24, 24, 24, d, (0.65, 0.52, 0.35), 0.0006, 0)
    vel = np.zeros_like(pos)
    vel[:, 1] = -1.0
    cfg.particle_count = len(pos)
    V, F = scenes.icosphere(3, 0.2, (0.8, 0.3, 0.5))
    anchors = np.argsort(V[:, 1], kind="stable")[:16]
    return cfg, pos, vel, V, F, anchors


def test_coupled_frames(have_gpu):
    cfg, pos, vel, V, F, anchors = small_c1()
    prm, kring, band = fsi.c1_deform_params()
    prm.control_threshold = 0.05
    prm.control_threshold_low = 0.03
    scene = fsi.CoupledScene(cfg, pos, vel, V, F, anchors, 0.0125, prm, band, kring=kring, incremental=True)
    moved_any = False
    for _ in range(12):
        forces, moved = scene.frame()
        moved_any |= moved
    assert scene.contacts > 0 and np.abs(forces).max() > 0
    assert moved_any and scene.refactors > 0
    Vd = scene.deform.vertices()
    disp = np.linalg.norm(Vd - V, axis=1)
    assert disp.max() > 1e-4
    assert disp.max() <= prm.max_total_disp * (1 + 1e-6)
    assert np.abs(Vd[anchors] - V[anchors]).max() < 1e-12
    # the collision SDF is the deformed mesh's: zero on its vertices (up to
    # trilinear interpolation of a 0.0125 grid), not on the rest vertices that moved
    d_def = scene.sdf.sample(Vd.astype(np.float32))
    assert np.abs(d_def).max() < 0.25 * 0.0125
    far = disp > 0.5 * 0.0125
    if far.any():
        d_rest = scene.sdf.sample(V[far].astype(np.float32))
        assert np.abs(d_rest).max() > 0.25 * 0.0125
    assert scene.fluid.check_finite() == 0
