"""The multi-scene engine against one single-scene handle per scene.

Every scene of a batch must evolve exactly as a PBFluids with the same
configuration: same segmented sort and cell table, same neighbour visitation,
same per-pair arithmetic.  Positions and velocities are compared after
several full steps; the tolerance (1e-6*h on positions, 1e-5 relative on
velocities) only absorbs FP32 contraction differences between separately
compiled kernels, and every option of the batch (block size, cell order,
persistent grid) must give bit-identical results to every other.
"""
import numpy as np
import pytest

import pbf_b200 as P
from pbf_b200 import batch as PB
from pbf_b200 import scenes as S

pytestmark = pytest.mark.gpu

SIZES = [1500, 3200, 700, 5000, 64]


def small_c3(sizes=SIZES, seed=11):
    cfg, sc = S.c3(seed=seed, count=len(sizes), sizes=sizes)
    cfg.particle_count = int(sum(sizes))
    return cfg, sc


def run_batch(cfg, sc, steps, options=()):
    b = PB.make_batch(cfg, sc)
    for opt, val in options:
        b.set_option(opt, val)
    for _ in range(steps):
        b.step()
    b.sync()
    return b.read_particles()


def test_batch_matches_one_handle_per_scene(have_gpu):
    cfg, sc = small_c3()
    got = run_batch(cfg, sc, 4)
    seq = PB.make_sequential(cfg, sc)
    off = 0
    h = cfg.h
    for (f, _), s in zip(seq, sc):
        for _ in range(4):
            f.step()
        ref = f.readbackParticles()
        mine = got[off:off + s["n"]]
        off += s["n"]
        dp = np.abs(mine["pos"] - ref["pos"]).max()
        vs = max(np.abs(ref["vel"]).max(), 1e-3)
        dv = np.abs(mine["vel"] - ref["vel"]).max() / vs
        assert dp <= 1e-6 * h, (s["n"], dp)
        assert dv <= 1e-5, (s["n"], dv)
    assert off == len(got)


@pytest.mark.parametrize("block", [64, 128, 256])
@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("bps", [0, 2])
def test_batch_options_are_bit_identical(have_gpu, block, order, bps):
    cfg, sc = small_c3()
    base = run_batch(cfg, sc, 2)
    got = run_batch(cfg, sc, 2, [(P.BOPT_BLOCK, block), (P.BOPT_ORDER, order), (P.BOPT_BLOCKS_PER_SM, bps)])
    assert np.array_equal(got["pos"], base["pos"]) and np.array_equal(got["vel"], base["vel"])


def test_graph_and_eager_agree(have_gpu):
    cfg, sc = small_c3()
    a = run_batch(cfg, sc, 3)
    b = run_batch(cfg, sc, 3, [(P.BOPT_USE_GRAPH, 0)])
    assert np.array_equal(a["pos"], b["pos"]) and np.array_equal(a["vel"], b["vel"])


def test_single_scene_batch_equals_handle(have_gpu):
    cfg, sc = small_c3(sizes=[4096])
    got = run_batch(cfg, sc, 3)
    (f, _sdf), = PB.make_sequential(cfg, sc)
    for _ in range(3):
        f.step()
    ref = f.readbackParticles()
    assert np.abs(got["pos"] - ref["pos"]).max() <= 1e-6 * cfg.h


def test_autotune_restores_state_and_reports_candidates(have_gpu):
    cfg, sc = small_c3()
    b = PB.make_batch(cfg, sc)
    b.step()
    before = b.read_particles()
    best, cands = b.autotune(2)
    after = b.read_particles()
    assert np.array_equal(before["pos"], after["pos"]) and np.array_equal(before["vel"], after["vel"])
    # 12 launch shapes of the hashed-bucket walk and the dense windows
    assert len(cands) == 13 and sorted(c["neighbour_mode"] for c in cands) == [4] * 12 + [8]
    assert best["ms_per_step"] == min(c["ms_per_step"] for c in cands)
    assert b.get_option(P.BOPT_BLOCK) == best["block"] and b.get_option(P.BOPT_ORDER) == best["order"]
    # stepping on with the tuned options continues the same trajectory
    ref = PB.make_batch(cfg, sc)
    for _ in range(3):
        ref.step()
    b.step()
    b.step()
    a = b.read_particles()
    r = ref.read_particles()
    assert np.array_equal(a["pos"], r["pos"])


@pytest.mark.parametrize("graph", [1, 0])
def test_dense_windows_are_bit_identical_to_buckets(have_gpu, graph):
    """Neighbour mode 8 (a dense cell window per scene, the passes over all
    scenes at once) gives the bits of the hashed-bucket walk, over steps in
    which the particles fall, splash and collide with each scene's sphere."""
    cfg, sc = small_c3(sizes=[1500, 3200, 700, 5000, 64, 9000])
    base = run_batch(cfg, sc, 6, [(P.BOPT_NEIGHBOUR_MODE, 4)])
    got = run_batch(cfg, sc, 6, [(P.BOPT_NEIGHBOUR_MODE, 8), (P.BOPT_USE_GRAPH, graph)])
    assert np.array_equal(got["pos"], base["pos"]) and np.array_equal(got["vel"], base["vel"])


def test_dense_windows_with_hash_collisions(have_gpu):
    """Small per-scene hash tables (different per scene) make many cells share
    buckets: those cells walk their scene's hashed buckets inside the dense
    passes, still bit-identical to the hashed-bucket walk."""
    cfg, sc = small_c3()
    for k, s in enumerate(sc):
        s["hash_size"] = [256, 4096, 1024, 2048, 64][k]
    base = run_batch(cfg, sc, 4, [(P.BOPT_NEIGHBOUR_MODE, 4)])
    got = run_batch(cfg, sc, 4, [(P.BOPT_NEIGHBOUR_MODE, 8)])
    assert np.array_equal(got["pos"], base["pos"]) and np.array_equal(got["vel"], base["vel"])


def test_dense_windows_with_drift_marks(have_gpu):
    """Particles placed 1.5 h beyond a wall are clamped back by more than the
    0.9 h drift bound; with small hash tables the queries they can reach
    through a colliding bucket are marked and walk the buckets for the rest
    of the substep: still the bits of the hashed-bucket walk."""
    cfg, sc = small_c3()
    for k, s in enumerate(sc):
        s["hash_size"] = 4096
        pos = s["pos"].copy()
        m = min(50, len(pos))
        pos[:m, 0] = s["bounds_max"][0] + 1.5 * cfg.h
        s["pos"] = pos
    base = run_batch(cfg, sc, 2, [(P.BOPT_NEIGHBOUR_MODE, 4)])
    got = run_batch(cfg, sc, 2, [(P.BOPT_NEIGHBOUR_MODE, 8)])
    assert np.array_equal(got["pos"], base["pos"]) and np.array_equal(got["vel"], base["vel"])


def test_dense_windows_match_one_handle_per_scene(have_gpu):
    cfg, sc = small_c3()
    got = run_batch(cfg, sc, 3, [(P.BOPT_NEIGHBOUR_MODE, 8)])
    off = 0
    for (f, _), s in zip(PB.make_sequential(cfg, sc), sc):
        f.set_option(1, 8)
        for _ in range(3):
            f.step()
        ref = f.readbackParticles()
        mine = got[off:off + s["n"]]
        off += s["n"]
        assert np.abs(mine["pos"] - ref["pos"]).max() <= 1e-6 * cfg.h


def test_neighbour_mode_option(have_gpu):
    cfg, sc = small_c3()
    b = PB.make_batch(cfg, sc)
    assert b.get_option(P.BOPT_NEIGHBOUR_MODE) == -1
    b.set_option(P.BOPT_NEIGHBOUR_MODE, 8)
    assert b.get_option(P.BOPT_NEIGHBOUR_MODE) == 8
    with pytest.raises(P.PBFError):
        b.set_option(P.BOPT_NEIGHBOUR_MODE, 6)


def test_dense_windows_refused_when_too_large(have_gpu):
    """A scene whose walls span more than 2^26 cells in all has no dense
    window: mode 8 is refused and the automatic choice walks the buckets."""
    cfg, sc = small_c3(sizes=[700, 1500])
    sc[1]["bounds_max"] = (400.0, 400.0, 400.0)  # 10^4 cells per axis at h = 0.04
    b = PB.make_batch(cfg, sc)
    with pytest.raises(P.PBFError):
        b.set_option(P.BOPT_NEIGHBOUR_MODE, 8)
    for _ in range(2):
        b.step()
    b.sync()
    got = b.read_particles()
    base = run_batch(cfg, sc, 2, [(P.BOPT_NEIGHBOUR_MODE, 4)])
    assert np.array_equal(got["pos"], base["pos"]) and np.array_equal(got["vel"], base["vel"])


def test_per_scene_io_and_errors(have_gpu):
    cfg, sc = small_c3()
    b = PB.make_batch(cfg, sc)
    assert b.info() == (len(sc), sum(SIZES))
    off = 0
    for k, s in enumerate(sc):
        assert b.scene_range(k) == (off, s["n"])
        one = b.read_particles(k)
        assert np.array_equal(one["pos"], s["pos"])
        off += s["n"]
    with pytest.raises(P.PBFError):
        b.scene_range(len(sc))
    with pytest.raises(P.PBFError):
        b.set_particles(0, P.make_particles(sc[1]["pos"]))  # wrong count
    with pytest.raises(P.PBFError):
        b.set_option(P.BOPT_BLOCK, 96)
    # replacing one scene's particles leaves the others untouched
    moved = P.make_particles(sc[2]["pos"] + np.float32(0.01))
    b.set_particles(2, moved)
    allp = b.read_particles()
    o2, n2 = b.scene_range(2)
    assert np.array_equal(allp["pos"][o2:o2 + n2], moved["pos"])
    assert np.array_equal(allp["pos"][:o2], np.concatenate([s["pos"] for s in sc[:2]]))
