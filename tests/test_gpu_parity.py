"""Parity of the sm_100a kernels (through the C ABI) with the FP64 oracle.

Integer work (hash keys, the stable sort permutation, the cell table, contact
compaction) must be bit-exact.  Floating-point stages are fed identical inputs
(the GPU's own state, converted to FP64) and must agree within FP32 rounding:
positions within 1e-5*h, other quantities relative to their scale as stated
in each assert.
"""
import ctypes as C

import numpy as np
import pytest

import oracle as O
import pbf_b200 as P
import pbfh as H
from pbf_b200 import scenes

pytestmark = pytest.mark.gpu

STAGE_FIXTURES = ["glsl_stages_plain.npz", "glsl_stages_scorr.npz", "glsl_stages_sdf.npz",
                  "glsl_stages_container.npz", "glsl_stages_apbf.npz"]


def make_fluid(z, mode=4):
    cfg = H.engine_cfg(z)
    fl = P.PBFluids(cfg)
    fl.set_option(1, mode)
    fl.setParticles(P.make_particles(z["pos0"], z["vel0"]))
    if "camera" in z:
        fl.setCameraPos(z["camera"])
    if "interaction" in z:
        fl.setInteraction(True, z["interaction"])
    sdf = None
    if "sdf_dist" in z:
        sdf = P.GridSDF(z["sdf_dist"], z["sdf_origin"], float(z["sdf_cell"]))
        fl.setSDFBoundary(sdf)
        fl.setSDFPadding(float(z["sdf_padding"]))
        fl.setSDFContainment(bool(z["sdf_containment"]))
    return fl, sdf


def gpu_sorted(fl, n):
    ids = fl.read_buffer(P.BUF_SORTED_IDS, np.uint32, n)
    xs = fl.read_buffer(P.BUF_XSTAR, np.float32, (n, 4))
    orig = np.zeros_like(xs)
    orig[ids] = xs
    return ids, xs, orig


# ---- sort / table -----------------------------------------------------------------
@pytest.mark.parametrize("n,bits,dist", [
    (1, 8, "rand"), (255, 8, "rand"), (4096, 17, "rand"), (4097, 17, "rand"), (100003, 22, "rand"),
    (1 << 20, 22, "rand"), (50000, 17, "equal"), (50000, 17, "sorted"), (50000, 17, "reverse"),
    (70001, 30, "few"), (20000, 32, "rand"), (30000, 1, "rand"), (9999, 9, "rand"),
])
def test_radix_sort_is_stable_and_bit_exact(have_gpu, n, bits, dist):
    rng = np.random.default_rng(n + bits)
    hi = (1 << bits) if bits < 32 else (1 << 32)
    if dist == "rand":
        keys = rng.integers(0, hi, size=n, dtype=np.uint64).astype(np.uint32)
    elif dist == "equal":
        keys = np.full(n, hi - 1, np.uint32)
    elif dist == "sorted":
        keys = np.sort(rng.integers(0, hi, size=n)).astype(np.uint32)
    elif dist == "reverse":
        keys = np.sort(rng.integers(0, hi, size=n))[::-1].astype(np.uint32)
    else:
        keys = rng.choice(np.array([0, 7, hi - 1, 12345 % hi], np.uint64), size=n).astype(np.uint32)
    sk, ids = P.sort_keys(keys, bits)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(ids, order.astype(np.uint32))
    assert np.array_equal(sk, keys[order])


def test_cell_table_bit_exact(have_gpu):
    rng = np.random.default_rng(5)
    for n, H_ in [(0, 1024), (1, 16), (5000, 1 << 12), (300000, 1 << 18)]:
        sk = np.sort(rng.integers(0, H_, size=n)).astype(np.uint32)
        t = P.build_table(sk, H_)
        ref = O.build_table(sk, H_) if n else np.full((H_, 2), -1, np.int32)
        assert np.array_equal(t, ref)
        assert (t[:, 1] - t[:, 0])[t[:, 0] >= 0].sum() == n


# A fixture with one config field overridden ("file.npz:field=value"): the
# s_corr exponent other than 4 takes the powf branch of the lambda pass's
# s_corr sum, which the fixtures' n = 4 never reaches.
STAGE_VARIANTS = ["glsl_stages_scorr.npz:n_corr=3", "glsl_stages_scorr.npz:n_corr=2.5"]


def load_stage_fixture(name):
    if ":" not in name:
        return H.load(name)
    base, mod = name.split(":")
    key, val = mod.split("=")
    z = H.load(base)
    z["cfg_" + key] = np.asarray(float(val), dtype=z["cfg_" + key].dtype)
    return z


# ---- substep stages against the oracle (GPU inputs -> FP64) ---------------------------
@pytest.mark.parametrize("name,mode", [(f, m) for m in (4, 8) for f in STAGE_FIXTURES + STAGE_VARIANTS])
def test_stages_match_oracle(have_gpu, name, mode):
    z = load_stage_fixture(name)
    fl, sdf = make_fluid(z, mode)
    p = H.oracle_params(z)
    S = H.oracle_sdf(z)
    L = O.lib()
    n = len(z["pos0"])
    h = p.cfg.h
    for st in (P.STAGE_PREDICT, P.STAGE_SORT, P.STAGE_TABLE, P.STAGE_REORDER):
        fl.run_stage(st)
    keys = fl.read_buffer(P.BUF_KEYS, np.uint32, n)
    sk = fl.read_buffer(P.BUF_SORTED_KEYS, np.uint32, n)
    table = fl.read_buffer(P.BUF_TABLE, np.int32, (p.cfg.hash_size, 2))
    ids, xs, xs_orig = gpu_sorted(fl, n)
    # keys from the GPU's own FP32 x*, its permutation and table: bit-exact
    assert np.array_equal(keys, O.keys_f32(xs_orig, h, p.cfg.hash_size - 1))
    osk, oids = O.stable_sort(keys, p.cfg.hash_size)
    assert np.array_equal(sk, osk) and np.array_equal(ids, oids)
    assert np.array_equal(table, O.build_table(osk, p.cfg.hash_size))
    # x* and v' against FP64 predict
    pos, vel = H.f64(z["pos0"]), H.f64(z["vel0"]).copy()
    x64 = np.zeros((n, 3))
    L.orc_predict(C.byref(p.p), n, pos.reshape(-1), vel.reshape(-1), x64.reshape(-1), None)
    assert np.abs(xs_orig[:, :3] - x64).max() < 1e-5 * h
    sv = fl.read_buffer(P.BUF_VPRED, np.float32, (n, 4))
    v_orig = np.zeros_like(sv)
    v_orig[ids] = sv
    assert np.abs(v_orig[:, :3] - vel).max() < 1e-6 * max(1.0, np.abs(vel).max())
    lod = None
    if p.p.apbf:
        lod_s = fl.read_buffer(P.BUF_LOD, np.uint32, n)
        lod = np.zeros(n, np.uint32)
        lod[ids] = lod_s
        olod = np.zeros(n, np.uint32)
        L.orc_lod(C.byref(p.p), n, H.f64(xs_orig[:, :3]).reshape(-1), olod)
        assert np.array_equal(lod, olod)
    lodp = lod.ctypes.data_as(C.c_void_p) if lod is not None else None
    iters = p.p.max_lod if p.p.apbf else p.cfg.solver_iterations
    tabf = table.reshape(-1)
    for it in range(1, iters + 1):
        _, _, x_in = gpu_sorted(fl, n)
        fl.run_stage(P.STAGE_LAMBDA, it)
        _, xl, xl_orig = gpu_sorted(fl, n)
        lam = np.zeros(n)
        rho = np.zeros(n)
        lam[:] = x_in[:, 3]  # inactive APBF particles keep their lambda
        L.orc_lambda(C.byref(p.p), n, H.f64(x_in[:, :3]).reshape(-1), ids, tabf, lodp, it, lam,
                     rho.ctypes.data_as(C.c_void_p))
        # lambda = -C / D with C = rho/rho0 - 1: the FP32 density carries ~1e-7
        # relative error, which C inherits absolutely (cancellation near rest)
        Cc = np.maximum(rho / p.p.rho0 - 1.0, -p.p.cohesion)
        big = np.abs(Cc) > 1e-3
        inv_d = np.abs(lam[big] / Cc[big]).max() if big.any() else 1.0 / p.p.eps
        tol = 2e-5 * np.abs(lam).max() + 1e-6 * inv_d * rho.max() / p.p.rho0
        assert np.abs(xl_orig[:, 3] - lam).max() <= tol, it
        rho_g = np.zeros(n, np.float32)
        rho_g[ids] = fl.read_buffer(P.BUF_RHO, np.float32, n)
        act = np.ones(n, bool) if lod is None else lod >= it
        assert np.abs(rho_g - rho)[act].max() < 2e-6 * rho.max()
        fl.run_stage(P.STAGE_DELTAP, it)
        _, _, xd_orig = gpu_sorted(fl, n)
        x64 = H.f64(xl_orig[:, :3]).copy()
        L.orc_deltap_apply(C.byref(p.p), S.ref() if S else None, n, x64.reshape(-1), H.f64(xl_orig[:, 3]), ids,
                           tabf, lodp, it, None)
        assert np.abs(xd_orig[:, :3] - x64).max() < 1e-5 * h, it
    # integrate
    _, _, xf_orig = gpu_sorted(fl, n)
    fl.run_stage(P.STAGE_INTEGRATE)
    pos_g = fl.read_buffer(P.BUF_POS, np.float32, (n, 4))
    vel_g = fl.read_buffer(P.BUF_VEL, np.float32, (n, 4))
    om_g = np.zeros((n, 4), np.float32)
    om_g[ids] = fl.read_buffer(P.BUF_OMEGA, np.float32, (n, 4))
    p64, v64, om = H.f64(z["pos0"]).copy(), H.f64(v_orig[:, :3]).copy(), np.zeros((n, 3))
    L.orc_integrate(C.byref(p.p), S.ref() if S else None, n, p64.reshape(-1), v64.reshape(-1),
                    H.f64(xf_orig[:, :3]).reshape(-1), ids, tabf, om.ctypes.data_as(C.c_void_p))
    assert np.abs(pos_g[:, :3] - p64).max() < 1e-5 * h
    assert np.abs(om_g[:, :3] - om).max() < 2e-5 * max(np.abs(om).max(), 1e-9)
    keep = np.ones(n, bool)
    if S is not None:
        xc = np.clip(H.f64(xf_orig[:, :3]), np.array(p.p.bmin[:]), np.array(p.p.bmax[:]))
        d, _ = S.query(xc)
        thr = -S.s.padding if S.s.containment else S.s.padding
        keep = np.abs(d - thr) > 1e-5 * S.s.cell
    vs = max(np.abs(v64).max(), 1.0)
    assert np.abs(vel_g[:, :3] - v64)[keep].max() < 2e-5 * vs
    # vorticity
    fl.run_stage(P.STAGE_VORTICITY)
    vel2 = fl.read_buffer(P.BUF_VEL, np.float32, (n, 4))
    v3 = H.f64(vel_g[:, :3]).copy()
    L.orc_vorticity(C.byref(p.p), n, H.f64(pos_g[:, :3]).reshape(-1), v3.reshape(-1), H.f64(om_g[:, :3]).reshape(-1),
                    ids, tabf)
    assert np.abs(vel2[:, :3] - v3).max() < 1e-5 * vs


@pytest.mark.parametrize("name", ["glsl_stages_plain.npz", "glsl_stages_apbf.npz"])
def test_first_substep_matches_reference_shaders_directly(have_gpu, name):
    """GPU substep vs the reference's own FP32 shader result (golden)."""
    z = H.load(name)
    fl, _ = make_fluid(z)
    n = len(z["pos0"])
    for st in (P.STAGE_PREDICT, P.STAGE_SORT, P.STAGE_TABLE, P.STAGE_REORDER):
        fl.run_stage(st)
    assert np.array_equal(fl.read_buffer(P.BUF_KEYS, np.uint32, n), z["pred_keys"])
    assert np.array_equal(fl.read_buffer(P.BUF_SORTED_IDS, np.uint32, n), z["sorted_grid"][:, 1])
    assert np.array_equal(fl.read_buffer(P.BUF_TABLE, np.int32, z["offsets"].shape), z["offsets"])
    cfg = H.engine_cfg(z)
    iters = cfg.max_lod if cfg.enable_apbf else cfg.solver_iterations
    for it in range(1, iters + 1):
        fl.run_stage(P.STAGE_LAMBDA, it)
        fl.run_stage(P.STAGE_DELTAP, it)
    fl.run_stage(P.STAGE_INTEGRATE)
    pos = fl.read_buffer(P.BUF_POS, np.float32, (n, 4))[:, :3]
    assert np.abs(pos - z["int_pos"]).max() < 1e-5 * cfg.h


def test_full_step_matches_oracle_smooth_regime(have_gpu):
    cfg, pos, vel = scenes.c0(16, seed=2)
    cfg.enable_scorr = 0
    cfg.particle_count = len(pos)
    vel = np.random.default_rng(9).uniform(-0.2, 0.2, pos.shape).astype(np.float32)
    fl = P.PBFluids(cfg)
    fl.setParticles(P.make_particles(pos, vel))
    fl.step()
    out = fl.readbackParticles()
    ocfg = O.FluidConfig()
    C.memmove(C.byref(ocfg), C.byref(cfg), C.sizeof(ocfg))
    p = O.Params(ocfg)
    p64, v64 = H.f64(pos).copy(), H.f64(vel).copy()
    O.step(p, p64, v64)
    err = np.abs(out["pos"] - p64).max()
    assert err <= 1e-5 * cfg.h, err / cfg.h
    assert np.abs(out["vel"] - v64).max() < 1e-3
    # predPos and the pad words come back as uploaded
    assert np.array_equal(out["pred_pos"], pos)


def test_graph_replay_and_repeat_runs_are_bit_identical(have_gpu):
    cfg, pos, vel = scenes.c0(16, seed=1)
    runs = []
    for graph in (False, True, True):
        fl = P.PBFluids(cfg)
        fl.setParticles(P.make_particles(pos, vel))
        fl.set_use_graph(graph)
        for _ in range(3):
            fl.step()
        runs.append(fl.readbackParticles())
        assert fl.kernel_launches() > 0
    for r in runs[1:]:
        assert np.array_equal(r["pos"], runs[0]["pos"]) and np.array_equal(r["vel"], runs[0]["vel"])


def test_empty_scene_and_errors(have_gpu):
    cfg, pos, vel = scenes.c0(8)
    fl = P.PBFluids(cfg)
    fl.setParticles(P.make_particles(pos[:0]))
    fl.step()  # no-op, as PBFluids.cpp:325
    assert len(fl.readbackParticles()) == 0
    with pytest.raises(P.PBFError):
        fl.run_stage(P.STAGE_LAMBDA, 1)
    fl.setParticles(P.make_particles(pos, vel))
    with pytest.raises(P.PBFError):
        fl.run_stage(P.STAGE_LAMBDA, 1)  # before the sort
    buf = np.zeros(3, P.PARTICLE_DTYPE)
    from pbf_b200 import _capi
    assert _capi.lib().pbf_read_particles(fl.handle, buf.ctypes.data_as(C.c_void_p), 3) == _capi.PBF_ERR_INVALID
    fl.step()
    assert fl.check_finite() == 0


# ---- SDF grid and contacts ---------------------------------------------------------------
def test_sdf_sampling_matches_oracle(have_gpu):
    z = H.load("glsl_stages_sdf.npz")
    g = P.GridSDF(z["sdf_dist"], z["sdf_origin"], float(z["sdf_cell"]))
    S = H.oracle_sdf(z)
    rng = np.random.default_rng(3)
    lo = np.array(z["sdf_origin"]) - 0.05
    hi = lo + np.array(z["sdf_dist"].shape) * float(z["sdf_cell"]) + 0.1
    pts = rng.uniform(lo, hi, size=(4000, 3)).astype(np.float32)
    d = np.empty(len(pts), np.float32)
    gr = np.empty((len(pts), 3), np.float32)
    from pbf_b200 import _capi
    _capi.check(_capi.lib().pbf_sample_sdf(g._h, pts.ctypes.data_as(C.c_void_p), len(pts),
                                           d.ctypes.data_as(C.c_void_p), gr.ctypes.data_as(C.c_void_p)))
    od, og = S.query(pts)
    assert np.abs(d - od).max() < 1e-6
    assert np.abs(gr - og).max() < 1e-3


def test_contact_filter_deterministic_and_exact(have_gpu):
    z = H.load("glsl_contacts.npz")
    fl, sdf = make_fluid(z)
    fl.filterContactCandidates(float(z["band"]))
    got = fl.readbackContactCandidates()
    S = H.oracle_sdf(z)
    pos = H.f64(z["pos0"])
    idx = np.zeros(len(pos), np.uint32)
    c = O.lib().orc_contact_filter(S.ref(), len(pos), pos.reshape(-1), float(z["band"]), idx)
    assert len(got) == c > 0
    # particle-index order, {pos, 0} and {vel, pad}
    assert np.array_equal(got["pos"][:, :3], z["pos0"][idx[:c]])
    assert np.all(got["pos"][:, 3] == 0)
    assert np.array_equal(got["vel"][:, :3], z["vel0"][idx[:c]])
    # band <= 0 is a no-op that keeps the previous list (PBFluids.cpp:195)
    fl.filterContactCandidates(0.0)
    assert len(fl.readbackContactCandidates()) == c


def test_sparse_clump_scene_agrees_between_modes(have_gpu):
    """Scattered particles and a dense clump (many cells without a clean
    neighbourhood, deep buckets): the dense-window passes (mode 8) fall back
    to the hashed buckets where they must and give the bucket walk's (mode 4)
    results bit for bit."""
    cfg, _, _ = scenes.c0(8)
    rng = np.random.default_rng(8)
    pos = rng.uniform(0.05, 0.95, size=(3000, 3)).astype(np.float32) * np.array([1.5, 0.9, 0.9], np.float32)
    pos[:1000] = pos[:1000] * 0.1 + 0.3  # and a dense clump
    vel = rng.uniform(-0.5, 0.5, size=pos.shape).astype(np.float32)
    cfg.enable_scorr = 0
    cfg.particle_count = len(pos)
    outs = []
    for mode in (4, 8):
        fl = P.PBFluids(cfg)
        fl.set_option(1, mode)
        fl.setParticles(P.make_particles(pos, vel))
        fl.step()
        outs.append(fl.readbackParticles())
    assert np.array_equal(outs[0]["pos"], outs[1]["pos"]) and np.array_equal(outs[0]["vel"], outs[1]["vel"])


def test_modes_agree_and_are_deterministic(have_gpu):
    """The masked bucket walk (4) and the dense-window runs (8) share the pair
    arithmetic and the visiting order: bit-identical.  Each mode is
    deterministic (two runs each), and the automatic choice is one of them."""
    cfg, pos, vel = scenes.c0(16, seed=4)
    cfg.enable_scorr = 0
    outs = {}
    for mode in (4, 4, 8, 8, -1):
        fl = P.PBFluids(cfg)
        fl.set_option(1, mode)
        fl.setParticles(P.make_particles(pos, vel))
        fl.step()
        o = fl.readbackParticles()
        if mode in outs:
            assert np.array_equal(outs[mode]["pos"], o["pos"]) and np.array_equal(outs[mode]["vel"], o["vel"])
        outs[mode] = o
    for m in (8, -1):
        assert np.array_equal(outs[4]["pos"], outs[m]["pos"]) and np.array_equal(outs[4]["vel"], outs[m]["vel"])


def test_removed_modes_are_refused(have_gpu):
    cfg, pos, vel = scenes.c0(8)
    fl = P.PBFluids(cfg)
    for mode in (0, 1, 2, 3, 5, 6, 7, 9):
        with pytest.raises(P.PBFError):
            fl.set_option(1, mode)


def _run_mode(cfg, pos, vel, mode, steps):
    fl = P.PBFluids(cfg)
    fl.set_option(1, mode)
    fl.setParticles(P.make_particles(pos, vel))
    for _ in range(steps):
        fl.step()
    return fl, fl.readbackParticles()


def _passes_per_step(cfg):
    return cfg.substep_iterations * (2 * cfg.solver_iterations + 1) + (1 if cfg.enable_vorticity else 0)


def test_dense_runs_agree_with_bucket_walk(have_gpu):
    """Mode 8 (x-runs of the dense cell window, relabelled data) visits the
    pairs of the hashed-bucket walk in the same order with the same pair
    arithmetic: bit-identical to mode 4 over three steps with s_corr on,
    although most particle passes take the runs."""
    cfg, pos, vel = scenes.c0(16, seed=6)
    cfg.particle_count = len(pos)
    _, a = _run_mode(cfg, pos, vel, 4, 3)
    fl, b = _run_mode(cfg, pos, vel, 8, 3)
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])
    walks, marked, unclean = fl.list_stats()
    assert walks < 0.5 * len(pos) * 3 * _passes_per_step(cfg)
    _, d = _run_mode(cfg, pos, vel, 8, 3)  # deterministic
    assert np.array_equal(b["pos"], d["pos"]) and np.array_equal(b["vel"], d["vel"])


def test_dense_window_change_and_particle_upload_between_steps(have_gpu):
    """In mode 8 the predict pass also writes each particle's window slot,
    which the relabelling of the same substep gathers.  Moving the walls (a
    new window) and uploading new particle state between steps make the
    relabelling derive the slots again; over a run with both, mode 8 stays
    bit-identical to mode 4."""
    cfg, pos, vel = scenes.c0(16, seed=4)
    cfg.particle_count = len(pos)
    out = []
    for mode in (4, 8):
        fl = P.PBFluids(cfg)
        fl.set_option(1, mode)
        fl.setParticles(P.make_particles(pos, vel))
        for _ in range(2):
            fl.step()
        hi = list(cfg.bounds_max)
        fl.setBounds(list(cfg.bounds_min), [hi[0] * 0.9, hi[1], hi[2] * 1.1], cfg.bound_damping)
        for _ in range(2):
            fl.step()
        mid = fl.readbackParticles()
        mid["pos"][:, 1] += np.float32(0.25 * cfg.h)
        fl.uploadParticles(mid)
        for _ in range(2):
            fl.step()
        out.append(fl.readbackParticles())
    assert np.isfinite(out[1]["pos"]).all()
    assert np.array_equal(out[0]["pos"], out[1]["pos"]) and np.array_equal(out[0]["vel"], out[1]["vel"])


def test_dense_particles_predicted_outside_the_window(have_gpu):
    """A particle whose predict-time cell lies outside the dense window (its
    velocity carries x* more than the window's margin past a wall) is
    relabelled into the overflow slot after every window slot; runs never
    reach it and the bucket walk finds it through the hash sort.  Over steps
    with many such particles, mode 8 stays bit-identical to mode 4."""
    cfg, pos, vel = scenes.c0(16, seed=5)
    cfg.particle_count = len(pos)
    vel = np.array(vel, dtype=np.float32, copy=True)
    rng = np.random.default_rng(5)
    pick = rng.choice(len(pos), 300, replace=False)
    # 40 m/s over a 1/120 s substep is 8 cells of h = 0.04, beyond the 6-cell margin
    vel[pick, :3] = rng.normal(0.0, 40.0, (len(pick), 3)).astype(np.float32)
    out = []
    for mode in (4, 8):
        fl = P.PBFluids(cfg)
        fl.set_option(1, mode)
        fl.setParticles(P.make_particles(pos, vel))
        for _ in range(3):
            fl.step()
        out.append(fl.readbackParticles())
    assert np.isfinite(out[1]["pos"]).all()
    assert np.array_equal(out[0]["pos"], out[1]["pos"]) and np.array_equal(out[0]["vel"], out[1]["vel"])


@pytest.mark.parametrize("hash_size", [32, 64, 4096])
def test_dense_runs_fall_back_on_hash_collisions(have_gpu, hash_size):
    """A small hash table makes neighbouring cells share buckets, which the
    reference then walks twice: the rows with such a collision within two
    cells walk the hashed buckets (32, 64: nearly all of them; 4096: some):
    bit-identical to mode 4.  With 32 buckets for 4,096 particles the window
    relabelling takes the radix sort instead of counting."""
    cfg, pos, vel = scenes.c0(16, seed=2)
    cfg.particle_count = len(pos)
    cfg.hash_size = hash_size
    cfg.enable_scorr = 0
    _, a = _run_mode(cfg, pos, vel, 4, 2)
    fl, b = _run_mode(cfg, pos, vel, 8, 2)
    walks, marked, unclean = fl.list_stats()
    assert unclean > 0 and walks > 0
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])


def test_dense_runs_drift_bound(have_gpu):
    """Particles placed 1.5 h beyond the +x wall are clamped back by more than
    the 0.9 h drift bound.  With a 4096-bucket table many cells have a
    same-bucket cell within a few cells: those particles mark the cells within
    their reach, whose queries walk the hashed buckets for the rest of the
    substep: bit-identical to mode 4."""
    cfg, pos, vel = scenes.c0(12, seed=3)
    cfg.substep_iterations = 1
    cfg.hash_size = 4096
    pos = pos.copy()
    pos[:50, 0] = cfg.bounds_max[0] + 1.5 * cfg.h
    cfg.particle_count = len(pos)
    _, a = _run_mode(cfg, pos, vel, 4, 1)
    fl, b = _run_mode(cfg, pos, vel, 8, 1)
    walks, marked, unclean = fl.list_stats()
    assert marked > 0 and walks > 0
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])


def test_automatic_mode_choice(have_gpu):
    """The default neighbour mode is chosen by size: the dense-window runs
    (mode 8, whose statistics report window cells) from 2^19 particles, the
    masked bucket walk (mode 4, no statistics) below; both bit-identical to
    the explicit modes."""
    cfg, pos, vel, sdf = scenes.c2(nx=128, ny=64, nz=64)  # 524,288 particles
    cfg.particle_count = len(pos)
    _, a = _run_mode(cfg, pos, vel, -1, 1)
    fl = P.PBFluids(cfg)
    fl.setParticles(P.make_particles(pos, vel))
    fl.step()
    assert fl.list_stats()[2] > 0
    _, b = _run_mode(cfg, pos, vel, 8, 1)
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])
    cfg, pos, vel = scenes.c0(16)
    cfg.particle_count = len(pos)
    fl = P.PBFluids(cfg)
    fl.setParticles(P.make_particles(pos, vel))
    fl.step()
    assert fl.list_stats() == (0, 0, 0)
    _, b = _run_mode(cfg, pos, vel, 4, 1)
    o = fl.readbackParticles()
    assert np.array_equal(o["pos"], b["pos"]) and np.array_equal(o["vel"], b["vel"])


def _capsule_scene():
    """A block of the C2 lattice (d = 0.005, h = 0.01) placed through the C2
    capsule obstacle: the first steps project many particles out of it, by
    several h, which exercises the drift marks of mode 8."""
    cfg, _, _, sdf = scenes.c2(nx=8, ny=8, nz=8)
    pos = scenes.lattice(48, 24, 48, 0.005, (1.08, 0.78, 0.38), 0.0002, 5)
    cfg.particle_count = len(pos)
    cfg.hash_size = scenes.hash_size_for(len(pos))
    return cfg, pos, np.zeros_like(pos), sdf


def _run_with_sdf(cfg, pos, vel, sdf, mode, steps, graph=False):
    fl = P.PBFluids(cfg)
    fl.set_option(1, mode)
    fl.set_use_graph(graph)
    fl.setParticles(P.make_particles(pos, vel))
    grid, origin, cell, pad = sdf
    obstacle = P.GridSDF(grid, origin, cell)
    fl.setSDFBoundary(obstacle)
    fl.setSDFPadding(pad)
    fl.setSDFContainment(False)
    for _ in range(steps):
        fl.step()
    out = fl.readbackParticles()
    return fl, out


def test_dense_runs_with_sdf_obstacle_and_graph(have_gpu):
    """Mode 8 against mode 4 in a scene whose particles start inside the
    capsule obstacle and are projected out by several h (drift marks, bucket
    walks near the obstacle), eager and replayed from a CUDA graph: bit-identical."""
    cfg, pos, vel, sdf = _capsule_scene()
    _, a = _run_with_sdf(cfg, pos, vel, sdf, 4, 5)
    fl, b = _run_with_sdf(cfg, pos, vel, sdf, 8, 5)
    _, c = _run_with_sdf(cfg, pos, vel, sdf, 8, 5, graph=True)
    for o in (b, c):
        assert np.array_equal(a["pos"], o["pos"]) and np.array_equal(a["vel"], o["vel"])
    walks, marked, unclean = fl.list_stats()
    assert walks > 0
    assert np.isfinite(b["pos"]).all()
