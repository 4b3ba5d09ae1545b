#!/usr/bin/env python3
"""Generate the golden fixtures in tests/golden from the reference's own code.

Run in a container that holds the reference tree, after ``make -C oracle ref``:

    python tests/golden/make_golden.py

Sources (all compiled from the reference by oracle/Makefile into oracle/_ref):
  * src/fluid/Kernels.cpp          -> kernels.npz     (poly6, spiky gradient)
  * src/fluid/NeighborSearch.cpp   -> neighbors.npz   (27-bucket neighbour lists)
  * resources/shaders/compute/*.glsl run on the CPU -> glsl_*.npz
    (per-dispatch state dumps and whole PBFluids::step results)

The fixtures are small seeded scenes; tests/test_oracle_golden.py checks the
FP64 oracle against them, which pins the oracle to the reference.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "realtime-fsi-engine_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle as O  # noqa: E402
from pbf_b200 import scenes  # noqa: E402

F32 = np.float32


derive_f32 = O.derive_f32


def to_oracle_cfg(cfg):
    c = O.FluidConfig()
    C.memmove(C.byref(c), C.byref(cfg), C.sizeof(c))
    return c


def small_scene(n_side=8, scorr=True, seed=0, hash_size=1 << 12):
    cfg, pos, vel = scenes.c0(n_side, seed)
    cfg.hash_size = hash_size
    cfg.enable_scorr = 1 if scorr else 0
    cfg.particle_count = len(pos)
    # non-uniform initial velocities so that XSPH and the curl are exercised
    vel = np.random.default_rng(seed + 100).uniform(-0.3, 0.3, size=pos.shape).astype(np.float32)
    return cfg, pos, vel


def sphere_grid(center, radius, cell):
    c = np.asarray(center, np.float64)
    lo = c - radius - 5 * cell
    hi = c + radius + 5 * cell
    dims = np.ceil((hi - lo) / cell).astype(int)
    xs = [lo[k] + np.arange(dims[k]) * cell for k in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    d = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2) - radius
    return d.astype(np.float32), lo, cell


def cfg_dict(cfg):
    return {k: np.array(getattr(cfg, k)) for k, _ in cfg._fields_}


def gen_kernels(out):
    L = O.ref_cpu()
    rng = np.random.default_rng(11)
    hs = np.array([0.04, 0.025, 0.01, 0.15], np.float32)
    rows = []
    for h in hs:
        r = rng.uniform(-1.2 * h, 1.2 * h, size=(400, 3)).astype(np.float32)
        r[:5] = 0.0
        r[5] = [h, 0, 0]
        r[6] = [0, 0, 1e-6]
        for v in r:
            g = np.zeros(3, np.float32)
            L.ref_grad_spiky(float(v[0]), float(v[1]), float(v[2]), float(h), g)
            w = L.ref_poly6(float(v[0]), float(v[1]), float(v[2]), float(h))
            rows.append([h, v[0], v[1], v[2], w, g[0], g[1], g[2]])
    np.savez_compressed(out, rows=np.array(rows, np.float32))


def gen_neighbors(out):
    L = O.ref_cpu()
    rng = np.random.default_rng(12)
    n = 1500
    pos = rng.uniform(-0.3, 0.3, size=(n, 3)).astype(np.float32)
    cell, H, cap = 0.08, 1 << 9, 160
    counts = np.zeros(n, np.int32)
    lists = np.full(n * cap, -1, np.int32)
    L.ref_neighbor_build(pos.reshape(-1), n, cell, H, counts, lists.ctypes.data_as(C.c_void_p), cap)
    assert counts.max() <= cap
    lists = lists.reshape(n, cap)
    lists = np.sort(np.where(lists < 0, np.iinfo(np.int32).max, lists), axis=1)
    np.savez_compressed(out, pos=pos, cell=np.float32(cell), hash_size=np.uint32(H), counts=counts, lists=lists)


def run_glsl(cfg, pos, vel, sdf=None, sort_mode=0, interaction=None, camera=(0, 0, 0), stages=False):
    d = derive_f32(cfg)
    S = O.GlslScene(d, to_oracle_cfg(cfg), pos, vel, sdf=sdf, sort_mode=sort_mode, parallel=False,
                    pre_integrate=True, interaction=interaction, camera=camera)
    rec = {}
    if stages:
        S.stage(1)
        rec["pred_xstar"] = S.solver[:, 0:3].copy()
        rec["pred_vel"] = S.vel.copy()
        rec["pred_keys"] = S.hg[:, 0].copy()
        S.stage(2)
        rec["sorted_grid"] = S.hg.copy()
        S.stage(3)
        rec["offsets"] = S.offsets.copy()
        if cfg.enable_apbf:
            S.stage(4)
            rec["lod"] = S.lod.copy()
        S.stage(5, 1)
        rec["lambda1"] = S.solver[:, 3].copy()
        rec["rho1"] = S.solver[:, 7].copy()
        S.stage(6, 1)
        rec["dp1"] = S.solver[:, 4:7].copy()
        S.stage(7, 1)
        rec["xstar1"] = S.solver[:, 0:3].copy()
        iters = cfg.max_lod if cfg.enable_apbf else cfg.solver_iterations
        for it in range(2, iters + 1):
            S.stage(5, it)
            S.stage(6, it)
            S.stage(7, it)
        rec["xstar_final"] = S.solver[:, 0:3].copy()
        rec["lambda_final"] = S.solver[:, 3].copy()
        S.stage(8)
        rec["int_pos"] = S.pos.copy()
        rec["int_vel"] = S.vel.copy()
        rec["int_omega"] = S.solver[:, 4:7].copy()
        if cfg.enable_vorticity:
            S.stage(9)
            rec["vort_vel"] = S.vel.copy()
    else:
        S.step()
        rec["pos"] = S.pos.copy()
        rec["vel"] = S.vel.copy()
        rec["grid"] = S.hg.copy()
        rec["offsets"] = S.offsets.copy()
    return rec


def gen_c0_scorr(out):
    """Config-0 first substep with s_corr: for each ensemble member the
    reference shaders' x* after every solver iteration and the committed
    positions, compared with FP64 on the same inputs (statistics only), plus
    member 0's committed FP32 positions for a direct GPU-vs-reference
    distance."""
    import c0_scorr as Z
    cfg, pos, vel = Z.scene()
    n, h = len(pos), float(cfg.h)
    iters = cfg.solver_iterations
    ref_stats = np.zeros((Z.N_MEMBERS, iters + 1, len(Z.STAT_NAMES)))
    ref_pos0 = None
    for m in range(Z.N_MEMBERS):
        pp = Z.member_inputs(pos, m)
        f64 = Z.fp64_stages(cfg, pp, vel)
        S = O.GlslScene(derive_f32(cfg), to_oracle_cfg(cfg), pp, vel, parallel=True)
        for st in (1, 2, 3):
            S.stage(st)
        for it in range(1, iters + 1):
            S.stage(5, it)
            S.stage(6, it)
            S.stage(7, it)
            ref_stats[m, it - 1] = Z.stats(S.solver[:, 0:3], f64[f"xstar{it}"], h)
        S.stage(8)
        ref_stats[m, iters] = Z.stats(S.pos, f64["pos"], h)
        if m == 0:
            ref_pos0 = S.pos.astype(np.float32).copy()
    np.savez_compressed(out, ref_stats=ref_stats, ref_pos0=ref_pos0,
                        pos0_sum=np.array([pos.astype(np.float64).sum(), (pos.astype(np.float64) ** 2).sum()]),
                        n=np.int64(n))


def gen_sdf_ref(out):
    """The reference's own SDFBoundary (src/fluid/SDFBoundary.cpp, compiled by
    oracle/Makefile) on an icosphere: the grid after buildFromMesh, after
    refitFromMesh of seeded moved vertices (build-time edge and vertex
    pseudo-normals kept), after buildFromMesh of the moved vertices (all
    pseudo-normals recomputed), and closestTriangle points at seeded
    queries."""
    V, F = scenes.icosphere(2, 0.2, (0.8, 0.3, 0.5))
    cell = 0.025
    rng = np.random.default_rng(21)
    V2 = V + rng.normal(0.0, 0.01, V.shape)
    V2[:20] += [0.0, 0.06, 0.0]  # a dent well beyond the noise
    R = O.RefSDF(V, F, cell)
    dims, org, c = R.info()
    grid = R.grid()
    pts = (rng.uniform(-0.3, 0.3, (500, 3)) + [0.8, 0.3, 0.5]).astype(np.float32)
    face, point = R.closest(pts)
    R.refit(V2)
    refit = R.grid()
    R2 = O.RefSDF(V2, F, cell)
    dims2, org2, _ = R2.info()
    np.savez_compressed(out, verts=V, faces=F.astype(np.int32), verts_moved=V2, cell=np.float64(cell), dims=dims,
                        origin=org, grid=grid, refit_grid=refit, rebuild_dims=dims2, rebuild_origin=org2,
                        rebuild_grid=R2.grid(), query=pts, closest_face=face, closest_point=point)


def save_scene(out, cfg, pos, vel, rec, sdf=None, extra=None):
    payload = dict(pos0=pos, vel0=vel, **{"cfg_" + k: v for k, v in cfg_dict(cfg).items()}, **rec)
    if sdf is not None:
        payload.update(sdf_dist=sdf.dist, sdf_origin=np.array(sdf.s.origin[:]), sdf_cell=np.float64(sdf.s.cell),
                       sdf_padding=np.float64(sdf.s.padding), sdf_containment=np.int32(sdf.s.containment))
    if extra:
        payload.update(extra)
    np.savez_compressed(out, **payload)


def main():
    if not O.have_ref():
        sys.exit("oracle/_ref not built: run `make -C oracle ref` first")
    gen_kernels(os.path.join(HERE, "kernels.npz"))
    gen_neighbors(os.path.join(HERE, "neighbors.npz"))

    # 1) stage-by-stage dumps, no s_corr (smooth regime), 10^3 block
    cfg, pos, vel = small_scene(10, scorr=False)
    save_scene(os.path.join(HERE, "glsl_stages_plain.npz"), cfg, pos, vel, run_glsl(cfg, pos, vel, stages=True))
    # 2) stage dumps with the benchmark's s_corr (k=0.1)
    cfg, pos, vel = small_scene(10, scorr=True, seed=3)
    save_scene(os.path.join(HERE, "glsl_stages_scorr.npz"), cfg, pos, vel, run_glsl(cfg, pos, vel, stages=True))
    # 3) whole step, radix shaders emulated, N not a multiple of 256, small H (collisions)
    cfg, pos, vel = small_scene(9, scorr=False, seed=4, hash_size=1 << 8)
    save_scene(os.path.join(HERE, "glsl_step_radix.npz"), cfg, pos, vel, run_glsl(cfg, pos, vel, sort_mode=1))
    # 4) SDF obstacle (sphere) and 5) container, stage dumps
    cfg, pos, vel = small_scene(10, scorr=False, seed=5)
    g, o, c = sphere_grid((0.1, 0.08, 0.1), 0.06, 0.01)
    sdf = O.Sdf(g, o, c, padding=0.005, containment=False)
    save_scene(os.path.join(HERE, "glsl_stages_sdf.npz"), cfg, pos, vel, run_glsl(cfg, pos, vel, sdf=sdf, stages=True),
               sdf=sdf)
    g, o, c = sphere_grid((0.1, 0.1, 0.1), 0.13, 0.01)
    sdf = O.Sdf(-g, o, c, padding=0.005, containment=True)
    save_scene(os.path.join(HERE, "glsl_stages_container.npz"), cfg, pos, vel,
               run_glsl(cfg, pos, vel, sdf=sdf, stages=True), sdf=sdf)
    # 6) APBF + mouse interaction, stage dumps
    cfg, pos, vel = small_scene(10, scorr=False, seed=6)
    cfg.enable_apbf, cfg.min_lod, cfg.max_lod, cfg.lod_max_dist = 1, 2, 5, 0.5
    cam = (0.0, 0.1, 0.0)
    ipos = (0.15, 0.15, 0.15)
    cfg.interaction_radius, cfg.interaction_strength = 0.1, 5.0
    save_scene(os.path.join(HERE, "glsl_stages_apbf.npz"), cfg, pos, vel,
               run_glsl(cfg, pos, vel, interaction=ipos, camera=cam, stages=True),
               extra=dict(camera=np.array(cam), interaction=np.array(ipos)))
    # 7) contact filter over a settled-ish state
    cfg, pos, vel = small_scene(10, scorr=False, seed=8)
    g, o, c = sphere_grid((0.1, 0.1, 0.1), 0.05, 0.01)
    sdf = O.Sdf(g, o, c, padding=0.005)
    S = O.GlslScene(derive_f32(cfg), to_oracle_cfg(cfg), pos, vel, sdf=sdf, parallel=False)
    S.c.contact_band = 0.03
    S.stage(10)
    cnt = int(S.count[0])
    save_scene(os.path.join(HERE, "glsl_contacts.npz"), cfg, pos, vel,
               dict(contacts=S.contacts[:cnt].copy(), band=np.float32(0.03)), sdf=sdf)
    # 8) the reference's mesh SDF: build, refit, rebuild, closest points
    gen_sdf_ref(os.path.join(HERE, "sdf_ref.npz"))
    # 9) config-0 first substep with s_corr, ensemble statistics
    gen_c0_scorr(os.path.join(HERE, "glsl_c0_scorr.npz"))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
