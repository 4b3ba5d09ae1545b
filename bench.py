#!/usr/bin/env python3
"""Headline benchmark: PBF particle-substeps/s on one B200 (or N replicas).

Workload (default): the large dam break, 4,194,304 particles (256x128x128
lattice, d=0.005, h=0.01), box 2x1x1, 1 substep per dt=1/120, 4 solver
iterations, static capsule SDF obstacle (r=0.1, axis z, x=1.2), FP32.  A
"step" is one PBFluids::step() (= one substep here) over the whole scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Timing: W untimed steps, then exactly K steps between CUDA events recorded on
the engine's stream, with a barrier + device synchronize on both sides; the
maximum over ranks is reported.  Each step replays the CUDA graph of the whole
step (pbf_set_use_graph); the per-pass times come from the same W + K steps
run again from the same state, launched one by one with events around every
pass (pbf_set_profiling).  The working set (~1.7 GB) is far larger than
the 126 MB L2, so no flush is needed between steps.  For N > 1 every rank steps
its own replica of the scene (the plain step does not shard; no collective).
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "realtime-fsi-engine_b200"))

METRIC = "particle-substeps/s"
# algorithmic bytes per particle and launch (payload only: vec3 = 12 B,
# scalar = 4 B; each pass reads its inputs and writes its outputs once); the
# cell table also clears its H buckets of 8 B each, 8 H / N per particle
ALGO_BYTES = {"predict_hash": 28, "radix_sort": 16, "cell_table": 12, "reorder": 64, "lambda": 16,
              "deltap_apply": 28, "integrate": 72, "vorticity": 48}


def algo_bytes(name, n, hash_size, mode=4):
    b = ALGO_BYTES.get(name, 0) * n
    if name == "cell_table":
        b += 8 * hash_size
    if name == "predict_hash" and mode == 8:
        b += 4 * n  # the window slot of each particle, written beside its hash key
    return b


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=["c2", "c0", "c1", "c3", "c4"], default="c2",
                    help="c2: 4M-particle dam break (headline); c0: 32k dam break; c1: coupled FSI frame; "
                         "c3: 64-scene batch vs the same scenes stepped one by one; "
                         "c4: differentiable step (adjoint cost and gradient checks)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="host seconds of the 64^3 sub-block CPU baseline")
    ap.add_argument("--ref-seconds", type=float, default=30.0,
                    help="host seconds of the reference arm's timed steps on the full scene")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="c2 only: skip the short C3 batch and C4 adjoint runs attached to the line")
    ap.add_argument("--mode", type=int, default=-1, choices=[-1, 4, 8],
                    help="neighbour passes: -1 automatic (default: 8 from 2^19 particles, else 4), 4 hashed "
                         "buckets in Morton thread order with per-bucket hit masks, 8 x-runs of a dense cell window")
    ap.add_argument("--sample", type=int, nargs=3, default=None, metavar=("NX", "NY", "NZ"),
                    help="smaller lattice of the same scene (profiling captures only)")
    return ap.parse_args()


# ---- distributed plumbing ------------------------------------------------------------
class Dist:
    def __init__(self, want):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", self.local))
            self.pg = dist
        if want != self.world and self.rank == 0:
            print(f"warning: --gpus {want} but WORLD_SIZE={self.world}", file=sys.stderr)

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=f"cuda:{self.local}")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.barrier()
            self.pg.destroy_process_group()


# ---- clocks ------------------------------------------------------------------------------
class Clocks:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.proc = None
        self.path = None
        try:
            import torch
            uuid = "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", uuid, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        smax = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[4 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ---- scenes ------------------------------------------------------------------------------
def workload_desc(name):
    if name == "c0":
        return "dam break 32^3 (32,768 particles, d=0.02, h=0.04, S=2, I=4)"
    return ("dam break 256x128x128 (4,194,304 particles, d=0.005, h=0.01, S=1 at dt=1/120, I=4, "
            "capsule SDF r=0.1 at x=1.2)")


def workload(name, sample=None):
    from pbf_b200 import scenes
    if name == "c0":
        cfg, pos, vel = scenes.c0(32)
        return cfg, pos, vel, None, workload_desc("c0")
    if sample:
        cfg, pos, vel, sdf = scenes.c2(nx=sample[0], ny=sample[1], nz=sample[2])
    else:
        cfg, pos, vel, sdf = scenes.c2()
    return cfg, pos, vel, sdf, workload_desc("c2")


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def traffic_summary(mode):
    """DRAM bytes per particle of the neighbour passes of one neighbour mode,
    from a committed ncu capture summary (profiles/traffic.json); the caller
    scales them to the workload."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json"))).get(str(mode), {})
    except Exception:
        return {}


# ---- CPU reference / baseline -------------------------------------------------------------------
def reference_side():
    """The oracle module and the scene generators, loaded without the engine
    package (the reference arm must not load or run any of the engine)."""
    import importlib.util
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    path = os.path.join(ROOT, "realtime-fsi-engine_b200", "pbf_b200", "scenes.py")
    spec = importlib.util.spec_from_file_location("pbf_scenes_standalone", path)
    S = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(S)
    S.FluidConfig = O.FluidConfig  # same layout as pbf_fluid_config
    return O, S


def cpu_reference_rate(budget_s, sample=(64, 64, 64), max_steps=50, warmup=0):
    """The reference's own compute shaders, compiled as C++ and run with
    OpenMP on the host cores (oracle/_ref), with the UBO derived by the
    reference's setParams float arithmetic (oracle.derive_f32), on the C2
    workload (`sample` = None) or a sub-block of its lattice; falls back to the
    FP64 oracle port when _ref is absent.  Steps run until `budget_s` seconds
    or `max_steps` steps, at least one."""
    O, S = reference_side()
    if sample:
        cfg, pos, vel, sdf = S.c2(nx=sample[0], ny=sample[1], nz=sample[2])
    else:
        cfg, pos, vel, sdf = S.c2()
    n = len(pos)
    grid, origin, cell, pad = sdf
    osdf = O.Sdf(grid, origin, cell, padding=pad, containment=False)
    cores = os.cpu_count() or 1
    what = (f"{sample[0]}x{sample[1]}x{sample[2]} sub-block of the 4M lattice ({n} particles, same d/h/constants/"
            "capsule)" if sample else f"the full C2 scene ({n} particles)")
    if O.have_ref():
        kind = "reference"
        scene = O.GlslScene(O.derive_f32(cfg), cfg, pos, vel, sdf=osdf, sort_mode=0, parallel=True,
                            pre_integrate=True)
        one = scene.step
    else:
        kind = "port"
        p = O.Params(cfg)
        p64, v64 = pos.astype(np.float64), vel.astype(np.float64)

        def one():
            O.step(p, p64, v64, sdf=osdf)
    for _ in range(warmup):
        one()
    steps = 0
    t0 = time.perf_counter()
    while True:
        one()
        steps += 1
        if time.perf_counter() - t0 > budget_s or steps >= max_steps:
            break
    dt = time.perf_counter() - t0
    rate = n * cfg.substep_iterations * steps / dt
    return {"value": rate, "unit": METRIC, "cores": cores, "kind": kind,
            "sample": f"{what}, {steps} steps in {dt:.1f} s after {warmup} warm-up, OpenMP over {cores} "
                      "host threads"}, cfg


def neighbour_work(pos, h, step_ms, passes, sample=100000, seed=0):
    """Neighbour work per step at a particle state (a host-side count after the timed
    runs, not timed): the candidates a query tests (the particles of the 27 cells
    around its own, the reference's bucket walk when no buckets collide) and the
    in-range pairs (r <= h, self excluded; a seeded sample of queries), per particle,
    and both per second over the `passes` neighbour passes of a step."""
    try:
        from scipy.ndimage import uniform_filter
        from scipy.spatial import cKDTree
    except ImportError:
        return None
    x = np.asarray(pos, np.float64)[:, :3]
    c = np.floor(x / h).astype(np.int64)
    c -= c.min(axis=0) - 1
    dims = c.max(axis=0) + 2
    occ = np.zeros((dims[2], dims[1], dims[0]), np.float64)
    np.add.at(occ, (c[:, 2], c[:, 1], c[:, 0]), 1.0)
    box = np.rint(uniform_filter(occ, size=3, mode="constant") * 27.0)
    cand = float((occ * box).sum() / len(x))
    rng = np.random.default_rng(seed)
    q = x[rng.choice(len(x), min(sample, len(x)), replace=False)]
    pairs = float(np.mean(cKDTree(x).query_ball_point(q, h, return_length=True)) - 1.0)
    per_s = len(x) * passes / (step_ms / 1e3)
    return {"candidates_per_particle": round(cand, 1), "in_range_pairs_per_particle": round(pairs, 2),
            "neighbour_passes_per_step": passes, "candidate_tests_per_s": cand * per_s,
            "pair_evaluations_per_s": pairs * per_s,
            "counted": f"on the state after the timed steps; pairs from {len(q)} seeded queries (k-d tree, r <= h)"}


def c2_config(desc, cfg, n):
    """The workload's config object, identical in both arms."""
    return {"workload": desc, "particles_per_gpu": n, "substeps": int(cfg.substep_iterations),
            "solver_iterations": int(cfg.solver_iterations), "hash_size": int(cfg.hash_size),
            "l2": "working set >> 126 MB L2 (no flush needed)"}


def run_reference(args):
    """The reference arm: the reference's shaders on the host cores, on the
    full 4,194,304-particle scene (one warm-up step, then steps until
    --ref-seconds; a few minutes at most).  Under torchrun only rank 0 runs."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.workload != "c2":
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm times the c2 workload only, "
                                                              f"not {args.workload}"}), flush=True)
        return
    full, cfg = cpu_reference_rate(args.ref_seconds, sample=None, max_steps=max(1, args.steps),
                                   warmup=min(args.warmup, 1))
    desc = workload_desc("c2")
    n = int(cfg.particle_count)
    line = {"impl": "reference", "metric": METRIC, "value": full["value"], "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": c2_config(desc, cfg, n), "parallelism": f"{full['cores']} host threads",
            "cpu_baseline": full,
            "e2e": {"value": full["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- GPU arm ------------------------------------------------------------------------------------------
def run_b200(args, dist):
    import torch

    import pbf_b200 as P
    dev = dist.local
    torch.cuda.set_device(dev)
    cfg, pos, vel, sdf, desc = workload(args.workload, sample=args.sample)
    if args.sample:
        desc = f"profiling sample {args.sample} of: " + desc
    n = len(pos)
    fl = P.PBFluids(cfg, device=dev)
    fl.set_option(1, args.mode)
    fl.setParticles(P.make_particles(pos, vel))
    obstacle = None
    if sdf is not None:
        grid, origin, cell, pad = sdf
        obstacle = P.GridSDF(grid, origin, cell, device=dev)
        fl.setSDFBoundary(obstacle)
        fl.setSDFPadding(pad)
        fl.setSDFContainment(False)
    stream = torch.cuda.ExternalStream(fl.stream(), device=dev)
    # timed: each step replays the CUDA graph of the whole step (captured on the
    # first warm-up step), no per-pass events
    start = fl.readbackParticles()
    fl.set_use_graph(True)
    for _ in range(args.warmup):
        fl.step()
    fl.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = Clocks(dev)
    l0 = fl.kernel_launches()
    mode = args.mode if args.mode >= 0 else (8 if n >= (1 << 19) else 4)
    ws0 = fl.list_stats() if mode == 8 else None
    e0.record(stream)
    for _ in range(args.steps):
        fl.step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    dist.barrier()
    clk = clocks.stop()
    launches = fl.kernel_launches() - l0
    ws1 = fl.list_stats() if ws0 is not None else None
    ms = e0.elapsed_time(e1)
    bad = fl.check_finite()
    # per-pass times: the same steps again from the same state, launched one
    # by one with CUDA events around every pass (the simulation is
    # deterministic, so the passes see the same particles as the timed run)
    fl.set_use_graph(False)
    fl.setParticles(start)
    for _ in range(args.warmup):
        fl.step()
    fl.sync()
    fl.set_profiling(True)
    fl.reset_pass_times()
    for _ in range(args.steps):
        fl.step()
    fl.sync()
    passes = fl.pass_times()
    fl.set_profiling(False)
    fl.set_use_graph(True)
    fl.step()  # re-capture the graph outside the e2e timing
    fl.sync()
    ms_max = dist.max(ms)
    subs = cfg.substep_iterations
    value = n * subs * args.steps * dist.world / (ms_max / 1e3)

    # e2e through the public API with host buffers: upload the state from
    # pinned memory, step, read the result back, every step
    pinned = torch.empty(n * 48, dtype=torch.uint8, pin_memory=True)
    host = pinned.numpy().view(P.PARTICLE_DTYPE)
    fl.readbackParticles(host)
    dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        fl.uploadParticles(host)
        fl.step()
        fl.readbackParticles(host)
    e2e_s = dist.max(time.perf_counter() - t0)
    e2e = {"value": n * subs * args.e2e_steps * dist.world / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": n * 48, "d2h_bytes_per_step": n * 48}
    # lambda and delta-p per iteration and integrate per substep, vorticity once per step
    nb_passes = (2 * cfg.solver_iterations + 1) * subs + (1 if cfg.enable_vorticity else 0)
    work = neighbour_work(host["pos"], cfg.h, ms_max / args.steps, nb_passes) if dist.rank == 0 else None

    # roofline of the dominant kernel (largest share of device time)
    pk = peaks()
    hbm = float(pk.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in pk else "fallback"
    per_pass = {}
    for name, (pms, cnt) in passes.items():
        if name == "step" or cnt == 0:
            continue
        per_launch = pms / cnt
        b = algo_bytes(name, n, cfg.hash_size, mode)
        per_pass[name] = {"ms_total": round(pms, 4), "launches": int(cnt), "ms_per_launch": round(per_launch, 5),
                          "share": round(pms / max(sum(v[0] for k, v in passes.items() if k != "step"), 1e-9), 4),
                          "algo_bytes_per_launch": b,
                          "gbs": round(b / (per_launch / 1e3) / 1e9, 1) if per_launch > 0 else None}
    dom = max(per_pass, key=lambda k: per_pass[k]["ms_total"]) if per_pass else None
    tr = traffic_summary(mode).get(dom) if dom else None
    roof = None
    if dom:
        ach = per_pass[dom]["gbs"]
        roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s",
                "frac": round(ach / hbm, 4) if ach else None,
                "traffic": (int(tr["bytes_per_particle"] * n) if tr else None),
                "peak_source": peak_src,
                "note": "neighbour passes are FP32-issue / L1 bound; algorithmic bytes = inputs + outputs once"}
    cb = None
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cb, _ = cpu_reference_rate(args.cpu_seconds)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": c2_config(desc, cfg, n), "neighbour_mode": mode,
            "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU",
            "roofline": roof, "cpu_baseline": cb, "e2e": e2e, "gpu_launches": int(launches), "clocks": clk,
            "passes": per_pass, "neighbour_work": work, "nonfinite_particles": int(bad), "impl": "b200"}
    if ws1 is not None:
        # pbf_list_stats before and after the timed steps (bucket walks, drift marks, unclean cells)
        line["walk_stats"] = {"before": list(ws0), "after": list(ws1)}
    del fl, obstacle
    if args.workload == "c2" and not args.no_extras and not args.sample:
        line.update(extra_workloads(args, dist))
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


def extra_workloads(args, dist):
    """Short runs of the two other figures the headline metric names, attached
    to the C2 line: the 64-scene batch against the same scenes stepped one by
    one (C3), and the adjoint/forward time ratio at 16 scenes with the
    smooth-variant gradient check against FP64 central differences (C4)."""
    import copy
    sub = copy.copy(args)
    sub.steps, sub.warmup, sub.e2e_steps = 5, 3, 2
    c3 = run_batch(sub, dist, emit=False)
    out = {"c3": {"value": c3["value"], "unit": METRIC, "ms_per_step": c3["ms_per_step"],
                  "sequential_ms_per_step": c3["sequential"]["ms_per_step"],
                  "speedup_vs_sequential": c3["speedup_vs_sequential"],
                  "max_pos_diff_vs_sequential": c3["max_pos_diff_vs_sequential"],
                  "particles": c3["config"]["particles_total"], "autotune_best": c3["autotune"]["best"],
                  "steps": sub.steps, "warmup": sub.warmup, "clocks": c3["clocks"],
                  "workload": c3["config"]["workload"]}}
    c4 = run_adjoint(sub, dist, emit=False, variants=("smooth",))
    gc = (c4.get("gradcheck") or {}).get("smooth (s_corr off, cohesion 0)") or {}
    out["c4"] = {"adjoint_over_forward_16_scenes": c4["value"], "costs": c4["costs"],
                 "gradcheck_smooth": {k: gc.get(k) for k in ("max_rel_gpu_vs_fd64", "max_rel_fp64_adjoint_vs_fd64",
                                                              "kink_rule", "directions_excluded",
                                                              "max_rel_gpu_vs_fd64_kept",
                                                              "median_rel_gpu_vs_fd64_kept",
                                                              "rel_vs_fp64_cpu_adjoint_velocity",
                                                              "rel_vs_fp64_cpu_adjoint_translation", "fd_eps")},
                 "steps": sub.steps, "warmup": sub.warmup, "clocks": c4["clocks"],
                 "workload": c4["config"]["workload"]}
    return out


def run_batch(args, dist, emit=True):
    """C3: 64 independent dam breaks in one multi-scene batch (one launch per
    pass, CUDA graph, autotuned launch shape), against the same scenes stepped
    one by one with one single-scene handle each.  With N ranks the scenes are
    partitioned by greedy size balance (no per-step exchange)."""
    import torch

    import pbf_b200 as P
    from pbf_b200 import batch as PB
    from pbf_b200 import scenes as S
    dev = dist.local
    torch.cuda.set_device(dev)
    cfg, allsc = S.c3()
    parts = PB.partition_scenes([s["n"] for s in allsc], dist.world)
    mine = [allsc[k] for k in parts[dist.rank]]
    n = sum(s["n"] for s in mine)
    n_all = sum(s["n"] for s in allsc)
    subs = cfg.substep_iterations
    b = PB.make_batch(cfg, mine, dev)
    best, cands = b.autotune(3)
    stream = torch.cuda.ExternalStream(b.stream(), device=dev)
    for _ in range(args.warmup):
        b.step()
    b.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = Clocks(dev)
    l0 = b.kernel_launches()
    e0.record(stream)
    for _ in range(args.steps):
        b.step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    dist.barrier()
    clk = clocks.stop()
    launches = b.kernel_launches() - l0
    ms_max = dist.max(e0.elapsed_time(e1))
    value = n_all * subs * args.steps / (ms_max / 1e3)

    # the same scenes, one single-scene handle each, stepped one after the
    # other (each scene's step completes before the next scene's starts), in
    # the neighbour mode that is faster for them (the dense-window relabelling
    # of mode 8 costs launches that small scenes do not earn back)
    seq_by_mode = {}
    for m in (4, 8):
        seq = PB.make_sequential(cfg, mine, dev)
        for f, _ in seq:
            f.set_option(1, m)
            f.set_use_graph(True)
        for _ in range(args.warmup):
            for f, _ in seq:
                f.step()
                f.sync()
        dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            for f, _ in seq:
                f.step()
                f.sync()
        seq_by_mode[m] = (dist.max(time.perf_counter() - t0), seq)
    seq_mode = min(seq_by_mode, key=lambda m: seq_by_mode[m][0])
    seq_s, seq = seq_by_mode[seq_mode]
    seq_value = n_all * subs * args.steps / seq_s
    # accuracy: both forms advanced warmup + steps from the same state
    got = b.read_particles()
    dmax, off = 0.0, 0
    for (f, _), s in zip(seq, mine):
        ref = f.readbackParticles()
        dmax = max(dmax, float(np.abs(got["pos"][off:off + s["n"]] - ref["pos"]).max()))
        off += s["n"]
    dmax = dist.max(dmax)

    # e2e through the public API with host buffers
    pinned = torch.empty(n * 48, dtype=torch.uint8, pin_memory=True)
    host = pinned.numpy().view(P.PARTICLE_DTYPE)
    b.read_particles(P.BATCH_ALL, host)
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        b.set_particles(P.BATCH_ALL, host)
        b.step()
        b.read_particles(P.BATCH_ALL, host)
    e2e_s = dist.max(time.perf_counter() - t0)
    line = {"metric": METRIC + " (64-scene batch)", "value": value, "unit": METRIC, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "64 dam breaks, N_i ~ U[4096, 131072] seed 7, box U[0.8,1.6]^3, sphere SDF "
                                   "r ~ U[0.05,0.2], d=0.02, h=0.04, S=2, I=4, H=2^17 per scene",
                       "particles_total": n_all, "particles_this_rank": n, "scenes_per_rank": [len(p) for p in parts],
                       "parallelism": f"scenes sharded x{dist.world}" if dist.world > 1 else "single GPU",
                       "l2": "working set > 126 MB L2 (no flush needed)"},
            "autotune": {"best": best, "candidates": cands},
            "sequential": {"value": seq_value, "ms_per_step": seq_s * 1e3 / args.steps,
                           "form": "one PBFluids handle per scene (CUDA graph each), stepped one after another",
                           "mode": seq_mode,
                           "ms_per_step_by_mode": {str(m): v[0] * 1e3 / args.steps for m, v in seq_by_mode.items()}},
            "speedup_vs_sequential": value / seq_value,
            "max_pos_diff_vs_sequential": dmax,
            "e2e": {"value": n_all * subs * args.e2e_steps / e2e_s, "unit": METRIC, "h2d_bytes_per_step": n * 48,
                    "d2h_bytes_per_step": n * 48},
            "roofline": None, "cpu_baseline": None, "gpu_launches": int(launches), "clocks": clk, "impl": "b200"}
    if emit and dist.rank == 0:
        print(json.dumps(line), flush=True)
    del seq, seq_by_mode, b
    return line


def run_adjoint(args, dist, emit=True, variants=("smooth", "cohesion", "configured")):
    """C4: differentiable C0 scene (32,768 particles, 16 substeps x 4
    iterations in one step, sphere obstacle r=0.15).  Times the forward step,
    the recording forward and the backward on 1 scene and on 16 scenes in
    one batch (jitter seeds 0..15); checks the GPU gradient against FP64
    central differences (eps=1e-4, 8 seeded directions of the initial
    velocities) and against the FP64 CPU adjoint.  The gradient check runs
    with s_corr off: with s_corr as configured (k=0.1 at unit mass) the
    step's tangent map has a norm ~1e43 and no difference quotient converges,
    which the line reports as evidence."""
    import torch

    import pbf_b200 as P
    from pbf_b200 import adjoint as A
    from pbf_b200 import scenes as S
    dev = dist.local
    torch.cuda.set_device(dev)
    cfg, pos, vel, target, sphere, grid = S.c4()
    n = len(pos)

    def make(cfg_, copies):
        sc = [dict(n=n, bounds_min=tuple(cfg_.bounds_min), bounds_max=tuple(cfg_.bounds_max),
                   hash_size=cfg_.hash_size) for _ in range(copies)]
        b = P.Batch(cfg_, sc, dev)
        for k in range(copies):
            pk = pos if k == 0 else S.c0(32, seed=k)[1]
            b.set_particles(k, P.make_particles(pk, vel))
            g, o, c, pad = grid
            b.set_sdf_grid(k, g, o, c)
            b.set_sdf_mode(k, pad, False)
        return b

    def timed(b, fn, reps):
        st = torch.cuda.ExternalStream(b.stream(), device=dev)
        for _ in range(max(args.warmup, 1)):
            fn()
        b.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(st)
        for _ in range(reps):
            fn()
        e1.record(st)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    costs = {}
    clocks = Clocks(dev)
    for copies in (1, 16):
        b = make(cfg, copies)
        zeros = torch.zeros((b.total, 4), dtype=torch.float32, device=f"cuda:{dev}")
        g = torch.zeros_like(zeros)
        g[:, 0] = 1.0 / b.total
        outp, outv = torch.empty_like(zeros), torch.empty_like(zeros)
        fwd = timed(b, b.step, args.steps)
        rec = timed(b, b.forward_record, args.steps)
        b.forward_record()
        bwd = timed(b, lambda: b.backward(g.data_ptr(), zeros.data_ptr(), outp.data_ptr(), outv.data_ptr()),
                    args.steps)
        costs[copies] = {"forward_ms": fwd, "record_ms": rec, "backward_ms": bwd,
                         "adjoint_over_forward": bwd / fwd, "record_plus_backward_over_forward": (rec + bwd) / fwd,
                         "particles": b.total}
        del b
    clk = clocks.stop()
    ratio = costs[16]["adjoint_over_forward"]

    # gradient checks (rank 0 only; CPU FP64 oracle)
    checks = None
    if dist.rank == 0:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        def oracle_params(c):
            oc = O.FluidConfig()
            C.memmove(C.byref(oc), C.byref(c), C.sizeof(oc))
            return O.Params(oc)

        g_, o_, c_, pad_ = grid

        def L64(Po, v0):
            p = pos.astype(np.float64).copy()
            v = v0.copy()
            O.step(Po, p, v, sdf=O.Sdf(g_, o_, c_, padding=pad_))
            return ((p - target) ** 2).sum(1).mean(), p

        def gpu_grad(c):
            b = make(c, 1)
            p = torch.tensor(pos, dtype=torch.float32, device=f"cuda:{dev}", requires_grad=True)
            v = torch.tensor(vel, dtype=torch.float32, device=f"cuda:{dev}", requires_grad=True)
            t = torch.zeros((1, 3), dtype=torch.float32, requires_grad=True)
            pT, _ = A.step(b, p, v, t)
            L = ((pT - torch.tensor(target, dtype=torch.float32, device=f"cuda:{dev}")) ** 2).sum(1).mean()
            L.backward()
            return v.grad.cpu().numpy().astype(np.float64), t.grad.numpy()[0].astype(np.float64), float(L)

        def variant(scorr, cohesion):
            c = P.FluidConfig()
            C.memmove(C.byref(c), C.byref(cfg), C.sizeof(c))
            c.enable_scorr = scorr
            c.cohesion_strength = cohesion
            return c

        def against_fp64(c, fd_dirs):
            Po = oracle_params(c)
            gv, gt, _ = gpu_grad(c)
            v64 = vel.astype(np.float64)
            _, pT = L64(Po, v64)
            t0 = time.perf_counter()
            _, gv64, gt64, _, _ = O.adjoint_step(Po, pos.astype(np.float64), v64, gpos=2 * (pT - target) / n,
                                                 sdf=O.Sdf(g_, o_, c_, padding=pad_))
            out = {"fp64_cpu_adjoint_seconds": time.perf_counter() - t0,
                   "fp64_grad_norm": float(np.linalg.norm(gv64)),
                   "gpu_grad_norm": float(np.linalg.norm(gv)) if np.all(np.isfinite(gv)) else "non-finite (FP32 range)",
                   "sdf_translation_grad_gpu": gt.tolist(), "sdf_translation_grad_fp64": gt64.tolist()}
            if np.all(np.isfinite(gv)) and np.isfinite(out["fp64_grad_norm"]):
                out["rel_vs_fp64_cpu_adjoint_velocity"] = float(np.linalg.norm(gv - gv64) / np.linalg.norm(gv64))
                out["rel_vs_fp64_cpu_adjoint_translation"] = float(np.linalg.norm(gt - gt64) / np.linalg.norm(gt64))
            if fd_dirs:
                rng = np.random.default_rng(8)
                eps = 1e-4
                dirs = []
                for _ in range(fd_dirs):
                    u = rng.normal(size=v64.shape)
                    u /= np.linalg.norm(u)
                    fd = (L64(Po, v64 + eps * u)[0] - L64(Po, v64 - eps * u)[0]) / (2 * eps)
                    dirs.append({"fd64": fd, "gpu": float((gv * u).sum()), "fp64_adjoint": float((gv64 * u).sum())})
                for d in dirs:
                    d["rel_gpu"] = abs(d["gpu"] - d["fd64"]) / max(abs(d["fd64"]), 1e-300)
                    d["rel_fp64_adjoint"] = abs(d["fp64_adjoint"] - d["fd64"]) / max(abs(d["fd64"]), 1e-300)
                out.update(fd_eps=eps, directions=dirs, max_rel_gpu_vs_fd64=max(d["rel_gpu"] for d in dirs),
                           max_rel_fp64_adjoint_vs_fd64=max(d["rel_fp64_adjoint"] for d in dirs))
                # a direction along which the FP64 adjoint itself misses the FP64
                # difference quotient by more than 1e-3 crosses a kink (clamp,
                # contact or neighbour-set change) within +-eps: reported, then
                # left out of the kept figures (the rule of the GPU adjoint test)
                kept = [d["rel_gpu"] for d in dirs if d["rel_fp64_adjoint"] <= 1e-3]
                out.update(kink_rule="excluded where |fp64_adjoint - fd64| > 1e-3 |fd64|",
                           directions_excluded=len(dirs) - len(kept),
                           max_rel_gpu_vs_fd64_kept=max(kept) if kept else None,
                           median_rel_gpu_vs_fd64_kept=float(np.median(kept)) if kept else None)
            return out

        checks = {}
        if "smooth" in variants:
            checks["smooth (s_corr off, cohesion 0)"] = against_fp64(variant(0, 0.0), 8)
        if "cohesion" in variants:
            checks["s_corr off, cohesion 0.001"] = against_fp64(variant(0, 0.001), 0)
        if "configured" in variants:
            checks["as configured (s_corr k=0.1, cohesion 0.001)"] = against_fp64(cfg, 0)
        checks["note"] = ("cohesion 0.001 puts the max(C, -cohesion) kink inside the jittered lattice's density "
                          "fluctuations, where FP32 and FP64 take different branches; with s_corr k=0.1 at unit "
                          "mass the step's tangent map has a norm ~1e43 and no gradient is usable in any precision")
    line = {"metric": "adjoint/forward time ratio (16 scenes)", "value": ratio, "unit": "x", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": costs[16]["backward_ms"],
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "C0 dam break 32,768 particles, 16 substeps x 4 iterations, sphere r=0.15 at "
                                   "(0.78,0.32,0.32); x16 scenes (jitter seeds 0..15) in one batch",
                       "l2": "16-scene working set > 126 MB L2"},
            "costs": costs, "gradcheck": checks, "clocks": clk, "roofline": None, "cpu_baseline": None,
            "impl": "b200"}
    if emit and dist.rank == 0:
        print(json.dumps(line), flush=True)
    return line


def run_coupled(args, dist):
    """C1: 262,144 particles onto a deformable icosphere (subdivision 4, 2,562
    vertices, r=0.2, 16 lowest vertices anchored).  Each frame: GPU fluid step,
    GPU contact candidates and per-vertex forces, host Laplacian deformation
    (incremental hard-constraint factor), GPU LBVH refit and SDF recompute of
    the moved mesh.  Frames are timed end to end on the host clock (the host
    deformation is part of the frame)."""
    import torch

    from pbf_b200 import fsi
    from pbf_b200 import scenes as S
    dev = dist.local
    torch.cuda.set_device(dev)
    cfg, pos, vel, V, F, anchors = S.c1()
    prm, kring, band = fsi.c1_deform_params()
    scene = fsi.CoupledScene(cfg, pos, vel, V, F, anchors, 0.0125, prm, band, kring=kring, incremental=True,
                             device=dev)
    for _ in range(args.warmup):
        scene.frame()
    for k in scene.times:
        scene.times[k] = 0.0
    scene.refactors = 0
    l0 = scene.fluid.kernel_launches()
    dist.barrier()
    torch.cuda.synchronize(dev)
    clocks = Clocks(dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        scene.frame()
    torch.cuda.synchronize(dev)
    wall = dist.max(time.perf_counter() - t0)
    clk = clocks.stop()
    n = len(pos)
    subs = cfg.substep_iterations
    value = n * subs * args.steps * dist.world / wall
    disp = np.linalg.norm(scene.deform.vertices() - V, axis=1)
    nv = len(V)
    line = {"metric": METRIC + " (coupled FSI frame)", "value": value, "unit": METRIC, "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "C1: 64^3 lattice (262,144 particles, d=0.0125, h=0.025, S=2, I=4) onto an "
                                   "icosphere (subdivision 4, 2,562 v / 5,120 f, r=0.2, 16 anchors), SDF cell d, "
                                   "incremental hard-constraint deformation, SDF refit every moved frame",
                       "deform": {"stiffness": prm.stiffness, "max_displacement": prm.max_displacement,
                                  "max_total_disp": prm.max_total_disp, "restore_strength": prm.restore_strength,
                                  "control_threshold": prm.control_threshold,
                                  "control_threshold_low": prm.control_threshold_low, "contact_band": band},
                       "parallelism": f"replicas x{dist.world}" if dist.world > 1 else "single GPU"},
            "phases_ms_per_frame": {k: v * 1e3 / args.steps for k, v in scene.times.items()},
            "state": {"handles": scene.handles, "refactors": scene.refactors, "contacts": scene.contacts,
                      "max_vertex_displacement": float(disp.max())},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": nv * 24, "d2h_bytes_per_step": nv * 12 + 4,
                    "note": "the coupled frame is end to end: forces come back to the host, vertices go out"},
            "roofline": None, "cpu_baseline": None,
            "gpu_launches": int(scene.fluid.kernel_launches() - l0), "clocks": clk, "impl": "b200"}
    if dist.rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)  # host only: no process group, no GPU
        return
    dist = Dist(args.gpus)
    try:
        if args.workload == "c1":
            run_coupled(args, dist)
        elif args.workload == "c3":
            run_batch(args, dist)
        elif args.workload == "c4":
            run_adjoint(args, dist)
        else:
            run_b200(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
