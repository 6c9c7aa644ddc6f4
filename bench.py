#!/usr/bin/env python
"""Cloth XPBD benchmark: cloth vertex-substeps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]
                    [--workload uniform_batch|single_drape|uneven_batch|warm_start|hair_groom|
                                large_cloth_hair|mesh_floor|mesh_cloth] [--cloths C]
                    [--floor mesh|height_grid|box|none]
                    [--self-collision]

One step = one PhysicsWorld cloth frame for every cloth of the workload: a single batched
launch of the device solver (pxb_cloths_step) advancing each cloth by solve_cloth(h = 1/60,
4 substeps, 10 iterations). Default workload: the uniform batch, 1024 sheets of 64x64, seeded
synthetic scenes (physxcoopa_b200/scenes.py). Vertex-substeps = sum of particles x substeps x
steps.

  value    device-resident throughput: inputs in HBM, K steps timed with CUDA events on the
           library's own stream, max over ranks (weak scaling: each rank runs the full batch).
  e2e      the same steps through the public C-ABI as an engine frame uses it: per step the
           step inputs (per-cloth step records, colliders) go host->device from pinned memory
           and every cloth's particle positions plus per-cloth bounds/speed come back to
           pinned host memory.
  roofline shared-memory bound (the cloth lives in shared memory during a step): algorithmic
           bytes per launch = sum over cloths of (iterations x constraints x 68 B + particles x
           150 B) x substeps, over the measured per-launch duration, against the device's
           shared-memory bandwidth measured on the spot by pxb_measure_smem_bandwidth.
  cpu_baseline  the reference's own solve_cloth (oracle/_ref, compiled from the reference's
           headers) on a bounded sample of the workload on the host's cores, whole cloths per
           thread as the reference's serial dispatch solves them.

--workload warm_start is the learned warm start on the uneven batch: training rows recorded from
the plain 20-iteration solver on a separately seeded batch, the network trained (Adam, lr 1e-3),
then the same benchmark state stepped with 20 plain iterations and with the network plus 4
iterations; where a substep's residual (max |len / rest - 1| over the stretch constraints) still
exceeds that cloth's largest residual under the plain solver over the same steps, it keeps
iterating (4 at a time, residual checked after each block, at most 20 in all): equal residual,
cloth by cloth. The restart fallback (back to the prediction, 20 plain iterations) is reported
beside it. `value` is the warm-start
throughput, `plain` the plain one.

--workload mesh_cloth is the general-topology path: 1024 cloths built from a triangulated disc
(1261 particles each, no grid structure; pxb_host_cloth_make_mesh), each pinned at two rim points
and draped over a sphere.

--impl reference runs only that CPU implementation (rank 0; other ranks exit 0).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SPEC = "cloth vertex-substeps/s on 1 B200: plain XPBD vs NN warm-start at equal residual"
METRIC = SPEC
UNIT = "vertex-substeps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--workload", default="uniform_batch",
                    choices=["uniform_batch", "single_drape", "uneven_batch", "warm_start", "hair_groom",
                             "large_cloth_hair", "mesh_floor", "mesh_cloth"])
    ap.add_argument("--cloths", type=int, default=None)
    ap.add_argument("--self-collision", action="store_true",
                    help="turn ClothParams::self_collision on for every cloth of the workload")
    ap.add_argument("--floor", choices=["mesh", "height_grid", "box", "none"], default="mesh",
                    help="mesh_floor workload: the floor collider (height_grid: the same samples as "
                         "TriangleMesh::from_height_grid; box / none measure the mesh query's share)")
    ap.add_argument("--side", type=int, default=64, help="sheet side of the uniform batch")
    ap.add_argument("--rings", type=int, default=20,
                    help="mesh_cloth workload: rings of the disc mesh (1 + 3 rings (rings + 1) particles)")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--graph", action="store_true",
                    help="step through the captured CUDA graph (pxb_cloths_step_graph) instead of pxb_cloths_step")
    ap.add_argument("--variant", type=int, default=None,
                    help="fix the kernel variant (0/1/2) instead of autotuning")
    return ap.parse_args()


def build_scene(args, rank):
    sc = _build_scene(args, rank)
    if getattr(args, "self_collision", False):
        # ClothParams::self_collision on every cloth, at the builder's self_distance (0.6 x spacing)
        for c in sc.cloths:
            c.params.self_collision = 1
        sc.name += " (self-collision)"
    return sc


def _build_scene(args, rank):
    from physxcoopa_b200 import scenes
    if args.workload == "single_drape":
        return scenes.single_drape(seed=rank)
    if args.workload == "uniform_batch":
        return scenes.uniform_batch(n=args.cloths or 1024, side=args.side, seed=1 + rank)
    if args.workload == "mesh_floor":
        sc = scenes.mesh_floor_batch(n=args.cloths or 4096, side=25, seed=12 + rank,
                                     height_grid=args.floor == "height_grid")
        if args.floor in ("box", "none"):  # the same sheets on an analytic box floor, or on nothing
            from physxcoopa_b200.arrays import box, collider_array
            floor = collider_array([box((2.0, 2.0, 0.02), (0.0, 0.0, -0.02))]) if args.floor == "box" \
                else collider_array([])
            sc.colliders = [floor.copy() for _ in sc.cloths]
            sc.geometries = []
            sc.name += f" ({args.floor} floor)"
        return sc
    if args.workload == "mesh_cloth":
        return scenes.mesh_cloth_batch(n=args.cloths or 1024, rings=args.rings, seed=13 + rank)
    return scenes.uneven_batch(n=args.cloths or 4096, seed=2 + rank)


def workload_config(args, sc):
    return {"workload": sc.name, "cloths": len(sc.cloths), "vertices": sc.vertices,
            "substeps": sc.substeps, "iterations": sc.iterations, "h": sc.h,
            "compliance": "structural 0 / shear 1e-6 / bend 1e-4",
            "l2": "inputs larger than L2 (device state of the batch exceeds 126 MB)"
            if sc.vertices * 64 > 126e6 else "inputs fit in L2"}


# ------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.device)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------------------------------
# reference CPU implementation (oracle/_ref) on the host cores
# ------------------------------------------------------------------------------------------

def reference_cpu(sc, seconds_target=12.0, threads=None):
    """Times the reference's solve_cloth on a bounded sample of the workload. Returns a dict."""
    import ctypes as C
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _checkers as K
    from physxcoopa_b200 import _abi as A
    threads = threads or os.cpu_count() or 1
    kind = "reference" if K.ref_available() else "port"
    n_total = len(sc.cloths)

    # collider geometry under the ids the scene's colliders name
    gids = getattr(sc, "geometries_ids", None) or [k + 1 for k in range(len(sc.geometries))]
    for gid, g in zip(gids, sc.geometries):
        K.register_geometry(gid, g)

    def timed(sample, steps, nthreads):
        if kind == "reference":
            refs = [K.RefCloth.from_arrays(sc.cloths[i]) for i in sample]
            cols = [sc.colliders[i] for i in sample]
            flat = np.ascontiguousarray(np.concatenate(cols)) if cols else np.zeros(0, A.COLLIDER)
            offs = np.zeros(len(sample) + 1, np.uint32)
            offs[1:] = np.cumsum([len(c) for c in cols])
            srcs = [sc.sources[i] if sc.sources and sc.sources[i] is not None
                    else np.zeros(0, A.GRAVITY_SOURCE) for i in sample]
            sflat = np.ascontiguousarray(np.concatenate(srcs)) if srcs else np.zeros(0, A.GRAVITY_SOURCE)
            soffs = np.zeros(len(sample) + 1, np.uint32)
            soffs[1:] = np.cumsum([len(x) for x in srcs])
            handles = (C.c_void_p * len(refs))(*[r.h for r in refs])
            return K.ref().pxbref_bench_cloths(handles, len(refs), A.ptr(flat), A.ptr(offs),
                                               A.ptr(sflat), A.ptr(soffs), K.vec(sc.gravity),
                                               sc.substeps, sc.iterations, sc.h, steps, nthreads)
        # the C restatement, single-threaded
        t0 = time.perf_counter()
        for _ in range(steps):
            for i in sample:
                c = sc.cloths[i].copy()
                K.oracle_step_cloth(c, sc.colliders[i], sources=sc.sources[i] if sc.sources else None,
                                    substeps=sc.substeps, iterations=sc.iterations, h=sc.h)
        return time.perf_counter() - t0

    # calibrate on one cloth, one step, one thread
    probe = timed([0], 1, 1)
    per_cloth = max(probe, 1e-4)
    nthreads = threads if kind == "reference" else 1
    n_sample = int(min(n_total, max(nthreads, seconds_target * nthreads / per_cloth)))
    n_sample = max(1, (n_sample // nthreads) * nthreads) if n_sample >= nthreads else n_sample
    sample = list(range(n_sample))
    wall = timed(sample, 1, nthreads)
    steps = 1
    if wall < 0.5 * seconds_target and n_sample == n_total:
        steps = max(1, int(seconds_target / max(wall, 1e-3)))
        wall = timed(sample, steps, nthreads)
    verts = sum(len(sc.cloths[i].particles) for i in sample) * sc.substeps * steps
    return {"value": verts / wall, "unit": UNIT, "cores": nthreads, "kind": kind,
            "sample": f"{n_sample} of {n_total} cloths of the workload, {steps} step(s) each, "
                      f"{nthreads} host threads, {wall:.1f} s (reference solve_cloth -O2; the "
                      f"reference has one stretch compliance, so shear runs at the structural one)"
            if kind == "reference" else f"{n_sample} cloths, oracle port, 1 thread, {wall:.1f} s"}


# ------------------------------------------------------------------------------------------
# main
# ------------------------------------------------------------------------------------------

def bench_hair(args, ctx_factory):
    """65,536 strands x 32 particles (hair_groom): particle-substeps/s of solve_strands."""
    import torch
    from physxcoopa_b200 import scenes
    sc = scenes.hair_groom(n_strands=args.cloths or 65536)
    ctx = ctx_factory()
    sid = ctx.add_strands(sc.sets[0])
    pos, rot = sc.root_path(0)
    ctx.set_strand_roots(sid, pos, rot)
    col = sc.meta["colliders_at"](0)
    d, keep = ctx.make_strand_step([sid], [col], iterations=sc.iterations, substeps=sc.substeps, h=sc.h)
    for _ in range(max(args.warmup, 3)):
        ctx.step_strands_desc(d)
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(0)
    clocks.start()
    time.sleep(0.3)
    l0 = ctx.launch_count
    with torch.cuda.stream(stream):
        t0.record(stream)
        for _ in range(args.steps):
            ctx.step_strands_desc(d)
        t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = t0.elapsed_time(t1)
    units = sc.particles * sc.substeps
    value = units * args.steps / (ms * 1e-3)
    # end to end: per frame the roots go up, the step runs, positions come back
    n = len(sc.sets[0].particles)
    out = np.zeros(n, __import__("physxcoopa_b200._abi", fromlist=["A"]).PARTICLE)
    e0 = time.perf_counter()
    for f in range(max(3, args.steps // 2)):
        pos, rot = sc.root_path(f + 1)
        ctx.set_strand_roots(sid, pos, rot)
        ctx.step_strands([sid], [sc.meta["colliders_at"](f + 1)], iterations=sc.iterations)
        out = ctx.read_strand_particles(sid, n)
    e2e_s = (time.perf_counter() - e0) / max(3, args.steps // 2)
    line = {"metric": "hair particle-substeps/s", "value": value, "unit": "particle-substeps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded groom)",
            "config": {"workload": sc.name, "strands": len(sc.sets[0].strands), "particles": n,
                       "substeps": sc.substeps, "iterations": sc.iterations},
            "e2e": {"value": units / e2e_s, "unit": "particle-substeps/s",
                    "h2d_bytes_per_step": 64 * len(sc.sets[0].strands), "d2h_bytes_per_step": 48 * n},
            "gpu_launches": ctx.launch_count - l0, "clocks": clk}
    print(json.dumps(line))
    del keep
    ctx.close()
    return 0


def hbm_roofline(traffic, per_launch_ms):
    """The same launch against HBM: DRAM bytes per launch (ncu, profiles/) over its duration,
    against MEASURED_PEAKS.json's copy bandwidth. Shows the step is not HBM-bound."""
    if not traffic:
        return None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        src = "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError, KeyError):
        peak, src = 6650.0, "fallback 6.65 TB/s"
    achieved = traffic / (per_launch_ms * 1e-3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": src}


def bench_large(args, local_rank):
    """The large-cloth configuration: one 512 x 512 sheet (20 iterations, draped on a capsule,
    whole-GPU path) stepped together with the 65,536 x 32 groom (20 iterations, roots on a moving
    sphere). One step = one frame of both. Units: (cloth vertices + hair particles) x substeps."""
    import torch
    from physxcoopa_b200 import _abi as A
    from physxcoopa_b200 import runtime as R
    from physxcoopa_b200 import scenes
    from physxcoopa_b200.arrays import capsule, collider_array
    ctx = R.Context(local_rank)
    side = 512
    w = scenes.SPACING * (side - 1)
    h = R.HostCloth(side, side, w, w, center=(0.0, 0.0, 1.0), params=scenes.cloth_params(), jitter=1e-3, seed=5)
    h.pin_static((-w / 2, w / 2, 1.0), 0.3 * scenes.SPACING)
    h.pin_static((w / 2, w / 2, 1.0), 0.3 * scenes.SPACING)
    h.build_tethers()
    cloth = h.arrays()
    cap = collider_array([capsule(0.5, 0.45 * w, (0.0, 0.0, 0.3), axis=0)])
    cid = ctx.add_cloth(cloth)
    dc, keep_c = ctx.make_step([cid], [cap], iterations=20)
    hair = scenes.hair_groom(n_strands=args.cloths or 65536)
    sid = ctx.add_strands(hair.sets[0])
    pos, rot = hair.root_path(0)
    ctx.set_strand_roots(sid, pos, rot)
    ds, keep_s = ctx.make_strand_step([sid], [hair.meta["colliders_at"](0)], iterations=hair.iterations,
                                      substeps=hair.substeps, h=hair.h)
    W = max(args.warmup, 3)
    for _ in range(W):
        ctx.step_desc(dc)
        ctx.step_strands_desc(ds)
    ctx.synchronize()
    stream = torch.cuda.ExternalStream(ctx.stream)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    l0 = ctx.launch_count
    cloth_ms = 0.0
    with torch.cuda.stream(stream):
        t0.record(stream)
        for _ in range(args.steps):
            c0.record(stream)
            ctx.step_desc(dc)
            c1.record(stream)
            ctx.step_strands_desc(ds)
        t1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = ctx.launch_count - l0
    ms = t0.elapsed_time(t1) / args.steps
    cloth_last_ms = c0.elapsed_time(c1)
    n_cloth, n_hair = len(cloth.particles), len(hair.sets[0].particles)
    units = (n_cloth + n_hair) * 4
    # end to end: roots and colliders up, cloth positions and hair particles back, every frame
    out = np.zeros(3 * n_cloth, np.float32)
    e_steps = max(3, args.steps // 2)
    e0 = time.perf_counter()
    for f in range(e_steps):
        ctx.step_desc(dc)
        pos, rot = hair.root_path(f + 1)
        ctx.set_strand_roots(sid, pos, rot)
        ctx.step_strands([sid], [hair.meta["colliders_at"](f + 1)], iterations=hair.iterations)
        ctx.read_positions(np.array([cid], np.uint64), out)
        ctx.read_strand_particles(sid, n_hair)
    e2e_s = (time.perf_counter() - e0) / e_steps
    line = {"metric": METRIC, "value": units / (ms * 1e-3), "unit": "vertex-substeps/s (cloth vertices + hair particles)",
            "n_gpus": 1, "steps": args.steps, "warmup": W, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes)",
            "config": {"workload": f"large cloth {side}x{side} (20 iterations, capsule, whole-GPU path) + {hair.name}",
                       "cloth_vertices": n_cloth, "hair_particles": n_hair, "substeps": 4,
                       "cloth_iterations": 20, "hair_iterations": hair.iterations,
                       "cloth_ms_last_step": cloth_last_ms,
                       "l2": "cloth state (~18 MB) fits in L2; hair state 2.1 M particles x 48 B exceeds it"},
            "e2e": {"value": units / e2e_s, "unit": "vertex-substeps/s",
                    "h2d_bytes_per_step": 192 + 312 + 64 * len(hair.sets[0].strands) + 312,
                    "d2h_bytes_per_step": 12 * n_cloth + 40 * n_hair},
            "roofline": None, "cpu_baseline": None, "gpu_launches": launches, "clocks": clk}
    del keep_c, keep_s
    ctx.close()
    return line


def bench_warm(args, local_rank):
    """Learned warm start vs the plain 20-iteration solver at equal residual (see the module
    docstring). Returns the JSON line."""
    import torch
    from physxcoopa_b200 import _abi as A
    from physxcoopa_b200 import runtime as R
    from physxcoopa_b200 import scenes
    n = args.cloths or 4096
    plain_iters, warm_iters = 20, 4
    ctx = R.Context(local_rank)
    ctx.set_cloth_variant(0 if args.variant is None else args.variant)
    # --- training rows from the plain solver on a separately seeded batch -------------------
    t0 = time.perf_counter()
    tr = scenes.uneven_batch(n=min(512, n), seed=102)
    ids = [ctx.add_cloth(c) for c in tr.cloths]
    xs, ys = [], []
    rec_steps, want = 40, 2_000_000
    for step in range(rec_steps):
        x, y = ctx.record(ids, tr.colliders, sources=tr.sources, iterations=plain_iters, substep=step % 4)
        keep = np.random.default_rng(step).random(len(x)) < want / (rec_steps * max(len(x), 1))
        xs.append(x[keep])
        ys.append(y[keep])
    for i in ids:
        ctx.remove_cloth(i)
    X, Y = np.concatenate(xs), np.concatenate(ys)
    t_rec = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = ctx.mlp_train(X, Y, epochs=40, batch=8192, learning_rate=1e-3, seed=0)
    t_train = time.perf_counter() - t0

    sc = scenes.uneven_batch(n=n, seed=2)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))
    W = max(args.warmup, 3)

    def run(kind, taus=None, collect=False, e2e=False):
        """Steps a fresh copy of the benchmark batch: W plain warm-up steps, then args.steps of
        `kind`. Timed with CUDA events unless `collect`, which reads the per-step warm results
        (a host round trip per step) instead."""
        ids = [ctx.add_cloth(c) for c in sc.cloths]
        d, keep = ctx.make_step(ids, sc.colliders, sc.gravity, sc.sources, sc.substeps, plain_iters, sc.h)
        for _ in range(W):
            ctx.step_desc(d)
        ctx.synchronize()
        res = []
        t_a, t_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launch_count
        ids_np = np.ascontiguousarray(ids, np.uint64)
        out = torch.empty(3 * sc.vertices, dtype=torch.float32, pin_memory=True).numpy() if e2e else None
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            t_a.record(stream)
            for _ in range(args.steps):
                if kind == "plain":
                    ctx.step_desc(d)
                elif kind == "plain_residual":
                    ctx.step_warm_desc(d, warm_iterations=0)
                elif kind == "warm_restart":
                    ctx.step_warm_desc(d, warm_iterations=warm_iters, thresholds=taus)
                else:
                    ctx.step_warm_desc(d, warm_iterations=warm_iters, thresholds=taus, continue_iterations=True)
                if e2e:
                    ctx.read_positions(ids_np, out)
                if collect:
                    res.append(ctx.read_warm_results(ids))
            t_b.record(stream)
        torch.cuda.synchronize()
        ms = t_a.elapsed_time(t_b) / args.steps
        launches = ctx.launch_count - l0
        for i in ids:
            ctx.remove_cloth(i)
        del keep
        return ms, res, launches

    ms_plain, _, _ = run("plain")
    _, res_p, _ = run("plain_residual", collect=True)
    rp = np.stack([r["residual"] for r in res_p])
    taus = rp.max(0).astype(np.float32)
    _, res_w, _ = run("warm", taus, collect=True)
    rw = np.stack([r["residual"] for r in res_w])
    fb = float(sum(r["fallbacks"].sum() for r in res_w) / sum(r["substeps"].sum() for r in res_w))
    extra = float(sum(r["extra_iterations"].sum() for r in res_w) / sum(r["substeps"].sum() for r in res_w))
    ms_restart, _, _ = run("warm_restart", taus)
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    ms_w_total, _, launches = run("warm", taus)
    clk = clocks.stop()
    ms_e2e, _, _ = run("warm", taus, e2e=True)
    verts = sc.vertices * sc.substeps
    value = verts / (ms_w_total * 1e-3)
    plain_value = verts / (ms_plain * 1e-3)
    al = lambda x: (x + 255) & ~255
    n_col = sum(len(c) for c in sc.colliders)
    n_src = sum(0 if s is None else len(s) for s in (sc.sources or []))
    h2d = al(192 * n) + al(312 * max(n_col, 1)) + al(24 * max(n_src, 1)) + al(4 * n) + al(48 * n)
    d2h = 12 * sc.vertices + 16 * n
    cons = sum(len(c.stretch) + len(c.bend) for c in sc.cloths)
    iters_done = warm_iters + extra
    algo_bytes = sc.substeps * (iters_done * cons * 68 + sc.vertices * 150)
    smem_bw = ctx.measure_smem_bandwidth()
    achieved = algo_bytes / (ms_w_total * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": W,
        "ms_per_step": ms_w_total, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 solve, bf16 network (fp32 accumulation)", "data": "synthetic (seeded scenes)",
        "config": dict(workload_config(args, sc), workload=f"warm_start on {sc.name}", iterations=plain_iters,
                       warm_iterations=warm_iters, residual="max |len/rest - 1| over stretch constraints",
                       equal_residual="per cloth: fall back where the residual exceeds the plain solver's "
                                      "max residual for that cloth over the same steps"),
        "plain": {"value": plain_value, "ms_per_step": ms_plain, "residual_median": float(np.median(rp)),
                  "residual_max": float(rp.max())},
        "warm_start": {"speedup_vs_plain": value / plain_value, "fallback_rate": fb,
                       "fallback": "continue iterating from the warm state, 4 at a time, to the threshold "
                                   "or 20 iterations", "extra_iterations_per_substep": extra,
                       "restart_fallback": {"ms_per_step": ms_restart, "speedup_vs_plain": ms_plain / ms_restart,
                                            "note": "restart from the prediction with 20 plain iterations"},
                       "residual_median": float(np.median(rw)), "residual_max": float(rw.max()),
                       "training": {"rows": int(len(X)), "final_loss": loss, "record_s": t_rec, "train_s": t_train,
                                    "scenes": "uneven batch seed 102 (512 cloths), plain 20 iterations, "
                                              f"{rec_steps} steps"}},
        "e2e": {"value": verts / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "smem", "achieved": achieved, "peak": smem_bw / 1e9, "unit": "GB/s",
                     "frac": achieved * 1e9 / smem_bw, "traffic": None,
                     "peak_source": "measured on this GPU by pxb_measure_smem_bandwidth",
                     "kernel": "cloth_step_kernel (warm start)", "algorithmic_bytes_per_launch": algo_bytes},
        "cpu_baseline": None,
        "gpu_launches": launches,
        "clocks": clk,
    }
    ctx.close()
    return line


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        sc = build_scene(args, 0)
        res = []
        for _ in range(max(args.warmup, 0)):
            pass  # the reference has no warm-up state; each sample builds fresh cloths
        for _ in range(args.steps):
            res.append(reference_cpu(sc, seconds_target=8.0))
        value = statistics.median(r["value"] for r in res)
        cb = dict(res[0])
        cb["value"] = value
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scenes)",
                "config": workload_config(args, sc), "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    if args.workload == "hair_groom":
        from physxcoopa_b200 import runtime as R
        return bench_hair(args, lambda: R.Context(local_rank))
    if args.workload == "large_cloth_hair":
        if rank == 0:
            print(json.dumps(bench_large(args, local_rank)))
        return 0
    if args.workload == "warm_start":
        if rank == 0:
            print(json.dumps(bench_warm(args, local_rank)))
        return 0

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    from physxcoopa_b200 import runtime as R

    sc = build_scene(args, rank)
    ctx = R.Context(local_rank)
    if sc.geometries:
        from physxcoopa_b200 import scenes
        scenes.register_geometries(ctx, sc)
    ids = [ctx.add_cloth(c) for c in sc.cloths]
    d, keep = ctx.make_step(ids, sc.colliders, sc.gravity, sc.sources, sc.substeps,
                            sc.iterations, sc.h)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))

    tune = None
    if args.variant is None:
        best, ms = ctx.autotune(d, trials=2)
        tune = {"chosen_variant": best, "ms_per_step_by_variant": ms,
                "variants": "block-size cap 512 / 768 / 1024 threads"}
    else:
        ctx.set_cloth_variant(args.variant)
        tune = {"chosen_variant": args.variant, "fixed": True}
    step = ctx.step_graph_desc if args.graph else ctx.step_desc
    for _ in range(max(args.warmup, 3)):
        step(d)
    ctx.synchronize()
    smem_bw = ctx.measure_smem_bandwidth()
    if dist:
        dist.barrier()

    # --- device-resident timed region ----------------------------------------------------
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launch_count
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.synchronize()
    with torch.cuda.stream(stream):
        t_start.record(stream)
        for k in range(args.steps):
            ev[k][0].record(stream)
            step(d)
            ev[k][1].record(stream)
        t_end.record(stream)
    ctx.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = ctx.launch_count - launches0
    elapsed_ms = t_start.elapsed_time(t_end)
    per_launch_ms = statistics.mean(a.elapsed_time(b) for a, b in ev)
    if dist:
        t = torch.tensor([elapsed_ms, per_launch_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms, per_launch_ms = float(t[0]), float(t[1])

    verts_per_step = sc.vertices * sc.substeps
    value = world * verts_per_step * args.steps / (elapsed_ms * 1e-3)

    # --- roofline of the dominant kernel (shared memory) ----------------------------------
    cons = sum(len(c.stretch) + len(c.bend) for c in sc.cloths)
    algo_bytes = sc.substeps * (sc.iterations * cons * 68 + sc.vertices * 150)
    achieved = algo_bytes / (per_launch_ms * 1e-3) / 1e9
    peak = smem_bw / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"cloth_step_{args.workload}.json")
    if os.path.exists(prof):
        try:
            pj = json.load(open(prof))
            traffic = pj.get("dram_bytes_per_launch_full_workload")
        except (OSError, ValueError):
            traffic = None

    # --- end to end through the public API with host buffers -----------------------------
    import ctypes as C
    e2e_steps = args.e2e_steps or max(3, args.steps // 2)
    out = torch.empty(3 * sc.vertices, dtype=torch.float32, pin_memory=True)
    out_np = out.numpy()
    # pinned host buffers the pipelined read alternates between (frame k lands while k + 1 runs)
    outs_np = [out_np, torch.empty(3 * sc.vertices, dtype=torch.float32, pin_memory=True).numpy()]
    ids_np = np.ascontiguousarray(ids, np.uint64)
    from physxcoopa_b200 import _abi as A
    res_out = np.zeros(len(ids), A.FRAME_RESULT)
    # and for the per-cloth results (bounds, largest speed, time: 32 B per cloth)
    res_pinned = [torch.empty(8 * len(ids), dtype=torch.float32, pin_memory=True).numpy().view(A.FRAME_RESULT)
                  for _ in range(2)]
    # pxb_cloths_step uploads one staging block per step: per-cloth step records (192 B),
    # collider snapshots (312 B), gravity sources (24 B), the launch order (4 B) and the posed
    # convex hulls (16 B x (2 faces + 2 face-vertex entries) per distinct hull and pose), each
    # section padded to 256 B.
    al = lambda x: (x + 255) & ~255
    n_col = sum(len(c) for c in sc.colliders)
    n_src = sum(0 if s is None else len(s) for s in (sc.sources or []))
    hull_bytes = 0
    seen = set()
    gids = getattr(sc, "geometries_ids", None) or []
    for cols in sc.colliders:
        for c in cols:
            if int(c["type"]) == A.SHAPE_CONVEX_HULL and c["enabled"] and int(c["geometry"]):
                key = tuple(np.asarray(c[f]).tobytes() for f in ("geometry", "position", "orientation",
                                                                  "local_center", "local_rotation", "geometry_scale"))
                if key not in seen:  # one posed block per distinct hull and pose
                    seen.add(key)
                    g = sc.geometries[gids.index(int(c["geometry"]))]
                    hull_bytes += 16 * (2 * len(g.face_planes) + 2 * len(g.face_vertices))
    h2d = (al(192 * len(ids)) + al(312 * max(n_col, 1)) + al(24 * max(n_src, 1)) + al(4 * len(ids))
           + al(hull_bytes))
    d2h = 12 * sc.vertices + 32 * len(ids) + 4
    ctx.synchronize()
    if dist:
        dist.barrier()
    def timed_e2e(pipelined):
        """Per step: the step call (its inputs uploaded from pinned memory), every particle
        position and the per-cloth results read back to pinned host memory. Pipelined:
        pxb_cloths_read_positions_async / pxb_cloths_read_results_async, step k's read-back
        copied while step k + 1 is prepared and runs, every copy landed before the closing
        event; else the blocking pxb_cloths_read_positions / pxb_cloths_read_results."""
        ctx.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for k in range(e2e_steps):
                step(d)
                if pipelined:
                    ctx.read_positions_async(ids_np, outs_np[k % 2])
                    ctx.read_results_async(ids_np, res_pinned[k % 2])
                else:
                    ctx.read_positions(ids_np, out_np)
                    ctx.lib.pxb_cloths_read_results(ctx.h, A.ptr(ids_np), len(ids_np), A.ptr(res_out))
            if pipelined:
                ctx.wait_positions()
            e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t[0])
        return world * verts_per_step * e2e_steps / (ms * 1e-3)

    e2e_blocking = timed_e2e(False)
    e2e_value = timed_e2e(True)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = reference_cpu(sc)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes)",
            "config": dict(workload_config(args, sc), parallelism=f"independent cloth batches x{world}",
                           autotune=tune, launch="pxb_cloths_step_graph (captured CUDA graph)" if args.graph
                           else "pxb_cloths_step"),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "read_back": "pipelined: pxb_cloths_read_positions_async + pxb_cloths_read_results_async, "
                                 "each step's positions and results copied to pinned host memory while the "
                                 "next step is prepared and runs",
                    "blocking_value": e2e_blocking},
            "roofline": {"bound": "smem", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "measured on this GPU by pxb_measure_smem_bandwidth",
                         "kernel": "cloth_step_kernel", "per_launch_ms": per_launch_ms,
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "hbm": hbm_roofline(traffic, per_launch_ms)},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk,
            "spec_metric": SPEC,
        }
        print(json.dumps(line))
    del keep
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
