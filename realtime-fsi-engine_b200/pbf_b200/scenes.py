"""Seeded synthetic scenes of the benchmark configurations.

The reference publishes no datasets; every scene is generated here from a seed
(numpy PCG64), with the sizes and constants of the five benchmark
configurations:

  C0  dam break, 32x32x32 lattice, d=0.02, h=0.04, box 1.6x1x1, S=2, I=4
  C1  coupled FSI, 64^3 lattice, d=0.0125, h=0.025, icosphere (subdiv 4, r=0.2)
  C2  large dam break, 256x128x128 lattice, d=0.005, h=0.01, box 2x1x1, S=1, I=4,
      static capsule obstacle r=0.1 (axis z, x=1.2)
  C3  64 independent dam breaks, N_i ~ U[4096, 131072] (seed 7)
  C4  differentiable C0 scene, 16 substeps x 4 iterations, sphere r=0.15

Constants the configurations leave open are fixed here (cohesion 0.001,
damping 0.5, H = smallest power of two >= max(2^17, N), the C1 box height,
the C2 capsule's y and length, the C4 sphere centre).
"""
import math

import numpy as np

try:
    from ._capi import FluidConfig
except ImportError:
    # Loaded as a stand-alone file, outside the package (a CPU-only caller
    # that must not load the engine, such as the benchmark's reference arm):
    # the caller assigns a ctypes struct with pbf_fluid_config's layout.
    FluidConfig = None


def lattice_density(h, d):
    """Sum of poly6 over a perfect cubic lattice of spacing d, self included:
    the density a unit-mass particle sees at rest.  The reference has no mass
    parameter (rho = sum W, CS_ComputeLambdas.glsl:117,140), so "mass chosen
    so the lattice density equals rho0" is the same as rho0 = this sum."""
    r = int(math.ceil(h / d))
    s = 0.0
    coeff = 315.0 / (64.0 * math.pi * h ** 9)
    for i in range(-r, r + 1):
        for j in range(-r, r + 1):
            for k in range(-r, r + 1):
                r2 = (i * i + j * j + k * k) * d * d
                if r2 <= h * h:
                    s += coeff * (h * h - r2) ** 3
    return s


def hash_size_for(n, minimum=1 << 17):
    hsz = minimum
    while hsz < n:
        hsz <<= 1
    return hsz


def base_config(h, d, box, substeps, iters, dt, n, hash_size=None):
    c = FluidConfig()
    c.dt = dt
    c.gravity[:] = [0.0, -9.81, 0.0]
    c.h = h
    c.rho0 = lattice_density(h, d)
    c.solver_iterations = iters
    c.substep_iterations = substeps
    c.eps = 100.0
    c.particle_count = n
    c.spacing = d
    c.bounds_min[:] = [0.0, 0.0, 0.0]
    c.bounds_max[:] = list(box)
    c.bound_damping = 0.5
    c.hash_size = hash_size if hash_size else hash_size_for(n)
    c.enable_scorr = 1
    c.k_corr = 0.1
    c.n_corr = 4.0
    c.delta_q = 0.2
    c.cohesion_strength = 0.001
    c.enable_viscosity = 1
    c.viscosity = 0.01
    c.interaction_radius = 1.5
    c.interaction_strength = 25.0
    c.enable_vorticity = 1
    c.vorticity_epsilon = 0.0005
    c.enable_apbf = 0
    c.min_lod = 2
    c.max_lod = 7
    c.lod_max_dist = 15.0
    return c


def lattice(nx, ny, nz, d, origin, jitter, seed):
    """Block of nx*ny*nz particles at (i+0.5)d + origin + U(-jitter, jitter),
    x fastest (the spawnParticles loop order, src/main.cpp:178-183)."""
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    g = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64)
    pos = (g + 0.5) * d + np.asarray(origin, dtype=np.float64)
    if jitter > 0:
        rng = np.random.default_rng(seed)
        pos += rng.uniform(-jitter, jitter, size=pos.shape)
    return pos.astype(np.float32)


def c0(n_side=32, seed=0):
    d, h = 0.02, 0.04
    n = n_side ** 3
    cfg = base_config(h, d, (1.6, 1.0, 1.0), 2, 4, 1.0 / 60.0, n, 1 << 17)
    pos = lattice(n_side, n_side, n_side, d, (0.0, 0.0, 0.0), 0.001, seed)
    return cfg, pos, np.zeros_like(pos)


def icosphere(subdiv, radius, center):
    """Icosahedron subdivided `subdiv` times, projected to the sphere
    (subdiv 4: 2,562 vertices, 5,120 outward-oriented faces)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
         (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
         (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, dtype=np.float64) / np.linalg.norm(p) for p in v]
    faces = list(f)
    for _ in range(subdiv):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    V = np.array(verts) * radius + np.asarray(center, dtype=np.float64)
    F = np.array(faces, dtype=np.int32)
    return V, F


def c1(seed=0):
    d, h = 0.0125, 0.025
    n = 64 ** 3
    box = (1.6, 1.6, 1.0)
    cfg = base_config(h, d, box, 2, 4, 1.0 / 60.0, n, hash_size_for(n))
    pos = lattice(64, 64, 64, d, (0.4, 0.55, 0.1), 0.001 * d / 0.02, seed)
    V, F = icosphere(4, 0.2, (0.8, 0.3, 0.5))
    anchors = np.argsort(V[:, 1], kind="stable")[:16]
    return cfg, pos, np.zeros_like(pos), V, F, anchors


def capsule_grid(radius, a, b, cell):
    """Analytic capsule SDF sampled on the reference grid layout: origin =
    bbox - 5 cells, dims = ceil(span / cell), voxel i at origin + i*cell,
    index = x*dy*dz + y*dz + z (SDFBoundary.cpp:299-308,421-436)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    lo = np.minimum(a, b) - radius
    hi = np.maximum(a, b) + radius
    buf = 5.0 * cell
    origin = lo - buf
    span = (hi + buf) - origin
    dims = np.ceil(span / cell).astype(int)
    xs = [origin[k] + np.arange(dims[k]) * cell for k in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    P = np.stack([X, Y, Z], -1)
    ab = b - a
    t = np.clip(((P - a) @ ab) / (ab @ ab), 0.0, 1.0)
    closest = a + t[..., None] * ab
    dist = np.linalg.norm(P - closest, axis=-1) - radius
    return dist.astype(np.float32), origin, cell


C2_CAPSULE = dict(radius=0.1, a=(1.2, 0.85, 0.2), b=(1.2, 0.85, 0.8))


def c2(seed=0, nx=256, ny=128, nz=128):
    d, h = 0.005, 0.01
    n = nx * ny * nz
    cfg = base_config(h, d, (2.0, 1.0, 1.0), 1, 4, 1.0 / 120.0, n, hash_size_for(n))
    pos = lattice(nx, ny, nz, d, (0.0, 0.0, 0.0), 0.0002, seed)
    grid, origin, cell = capsule_grid(C2_CAPSULE["radius"], C2_CAPSULE["a"], C2_CAPSULE["b"], d)
    return cfg, pos, np.zeros_like(pos), (grid, origin, cell, d / 2.0)


def sphere_grid(radius, center, cell):
    """Analytic sphere SDF on the reference grid layout (as capsule_grid)."""
    c = np.asarray(center, np.float64)
    buf = 5.0 * cell
    origin = c - radius - buf
    dims = np.full(3, int(np.ceil((2.0 * (radius + buf)) / cell)))
    xs = [origin[k] + np.arange(dims[k]) * cell for k in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    dist = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - radius
    return dist.astype(np.float32), origin, cell


def block(n, d, box, jitter, seed):
    """n particles in a cubic-ish lattice block at the box corner: side
    ceil(cbrt n) cells in x and z (capped to the box), rows stacked in y, the
    top layer partial (x fastest, then z, then y)."""
    side = int(math.ceil(round(n ** (1.0 / 3.0), 9)))
    nx = max(1, min(side, int(box[0] / d) - 1))
    nz = max(1, min(side, int(box[2] / d) - 1))
    ny = int(math.ceil(n / (nx * nz)))
    if ny * d > box[1]:  # too tall for the box: spread over the whole floor
        nx = max(1, int(box[0] / d) - 1)
        nz = max(1, int(box[2] / d) - 1)
        ny = int(math.ceil(n / (nx * nz)))
    j, k, i = np.meshgrid(np.arange(ny), np.arange(nz), np.arange(nx), indexing="ij")
    g = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)[:n].astype(np.float64)
    pos = (g + 0.5) * d
    if jitter > 0:
        pos += np.random.default_rng(seed).uniform(-jitter, jitter, size=pos.shape)
    return pos.astype(np.float32)


def c3_sizes(seed=7, count=64):
    rng = np.random.default_rng(seed)
    return rng.integers(4096, 131072 + 1, size=count)


def c3(seed=7, count=64, sizes=None):
    """C3: `count` independent dam breaks sharing the C0 constants (d=0.02,
    h=0.04, S=2, I=4, H=2^17 per scene).  From one generator seeded `seed`:
    N_i ~ U[4096, 131072], box per axis ~ U[0.8, 1.6], sphere radius ~
    U[0.05, 0.2]; the sphere sits at (0.75 bx, 0.3 by, 0.5 bz), padding d/2.
    Returns (cfg, scenes), each scene a dict with n, bounds_min, bounds_max,
    pos, vel and sdf = (grid, origin, cell, padding)."""
    d, h = 0.02, 0.04
    rng = np.random.default_rng(seed)
    ns = rng.integers(4096, 131072 + 1, size=count) if sizes is None else np.asarray(sizes)
    boxes = rng.uniform(0.8, 1.6, size=(count, 3))
    radii = rng.uniform(0.05, 0.2, size=count)
    cfg = base_config(h, d, (1.6, 1.0, 1.0), 2, 4, 1.0 / 60.0, int(ns.sum()), 1 << 17)
    scenes = []
    for k in range(count):
        box = boxes[k]
        pos = block(int(ns[k]), d, box, 0.001, seed * 1000 + k)
        center = (0.75 * box[0], 0.3 * box[1], 0.5 * box[2])
        grid, origin, cell = sphere_grid(float(radii[k]), center, d)
        scenes.append(dict(n=int(ns[k]), bounds_min=(0.0, 0.0, 0.0), bounds_max=tuple(float(v) for v in box),
                           hash_size=1 << 17, pos=pos, vel=np.zeros_like(pos),
                           sdf=(grid, origin, cell, d / 2.0), radius=float(radii[k]), center=center))
    return cfg, scenes


def c4(seed=0):
    """C4: the C0 block with 16 substeps x 4 iterations in one step; target =
    lattice + (0.3, 0, 0.1) + N(0, 0.01) (seed 1); a sphere obstacle r=0.15
    centred at (0.78, 0.32, 0.32), touching the block's +x face so that its
    translation has a gradient within the step.  Returns cfg, pos, vel,
    target, sphere and the sphere's SDF grid (grid, origin, cell, padding)."""
    cfg, pos, vel = c0(32, seed)
    cfg.substep_iterations = 16
    rng = np.random.default_rng(1)
    target = pos.astype(np.float64) + np.array([0.3, 0.0, 0.1]) + rng.normal(0.0, 0.01, size=pos.shape)
    sphere = dict(radius=0.15, center=(0.78, 0.32, 0.32))
    d = 0.02
    grid, origin, cell = sphere_grid(sphere["radius"], sphere["center"], d)
    return cfg, pos, vel, target, sphere, (grid, origin, cell, d / 2.0)
