"""Seeded scenes shared by the adjoint tests (oracle-only and GPU).

A small dam-break block (nside^3 lattice, d=0.02, h=0.04, C0 constants) in a
0.5^3 box with random initial velocities N(0, 0.3) and, optionally, a sphere
SDF obstacle (r=0.08) the block runs into; the loss is the mean squared
distance of the final positions to a jittered translated copy of the start.
"""
import ctypes as C

import numpy as np

import oracle as O
from pbf_b200 import scenes as S


def setup(nside=8, subs=1, iters=1, sdf=True, scorr=True, visc=True, vort=True, seed=0, cohesion=None):
    """Returns (cfg, oracle params, pos, vel, grid, target); grid is
    (dist, origin, cell, padding) or None."""
    d, h = 0.02, 0.04
    n = nside ** 3
    cfg = S.base_config(h, d, (0.5, 0.5, 0.5), subs, iters, 1 / 60, n, 1 << 12)
    cfg.enable_scorr, cfg.enable_viscosity, cfg.enable_vorticity = int(scorr), int(visc), int(vort)
    if cohesion is not None:
        cfg.cohesion_strength = cohesion
    pos = S.lattice(nside, nside, nside, d, (0.1, 0.05, 0.1), 0.001, seed).astype(np.float64)
    rng = np.random.default_rng(seed + 1)
    vel = rng.normal(0, 0.3, pos.shape)
    oc = O.FluidConfig()
    C.memmove(C.byref(oc), C.byref(cfg), C.sizeof(oc))
    P = O.Params(oc)
    grid = None
    if sdf:
        g, origin, cell = S.sphere_grid(0.08, (0.2, 0.12, 0.2), d)
        grid = (g, origin, cell, d / 2)
    target = pos + np.array([0.05, 0, 0.02]) + rng.normal(0, 0.01, pos.shape)
    return cfg, P, pos, vel, grid, target


def mk_sdf(grid, t):
    if grid is None:
        return None
    g, o, c, pad = grid
    return O.Sdf(g, np.asarray(o) + t, c, padding=pad)


def loss(P, pos, vel, grid, t, target):
    """FP64 oracle loss (mean squared distance of final positions to target)
    with the final state."""
    p, v = pos.copy(), vel.copy()
    O.step(P, p, v, sdf=mk_sdf(grid, t))
    return ((p - target) ** 2).sum(1).mean(), p, v
