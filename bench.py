#!/usr/bin/env python
"""Cloth XPBD benchmark: cloth vertex-substeps/s on B200, plain XPBD and the learned warm start.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mine|reference]
                    [--workload uneven_batch|uniform_batch|single_drape|warm_start|hair_groom|
                                large_cloth_hair|mesh_floor|mesh_cloth] [--cloths C]
                    [--no-warm] [--shear-compliance X] [--floor mesh|height_grid|box|none]
                    [--self-collision]

Default workload: the uneven batch, 4096 sheets with sides drawn U{16..128}, 1-3 sphere / capsule /
oriented-box colliders each, half of them under a point gravity source, 4 substeps x 10 iterations,
seeded synthetic scenes (physxcoopa_b200/scenes.py; no dataset exists for this path). One step =
one PhysicsWorld cloth frame for every cloth: solve_cloth(h = 1/60) on each, batched in one
pxb_cloths_step call. Vertex-substeps = sum of particles x substeps x steps.

Compliances: structural and shear constraints at the one stretch compliance the reference's
ClothParams holds (0), bend 1e-4, in both arms; --shear-compliance X gives the shear constraints
their own compliance through the library's per-batch extension (no reference counterpart).

  value    device-resident throughput: inputs in HBM, K steps timed with CUDA events on the
           library's stream, max over ranks.
  e2e      the same steps through the public C-ABI as an engine frame uses it: per step the step
           inputs (per-cloth step records, colliders, sources) go host->device from pinned memory,
           every particle position and the per-cloth bounds / speed come back to pinned host
           memory (pipelined one frame, as a renderer consumes them).
  warm_start  the learned warm start on the same batch: a network trained on rows recorded from
           the plain 20-iteration solver on a separately seeded batch (the library's own kernels,
           Adam lr 1e-3), then the batch stepped with 20 plain iterations and with the network plus
           4 iterations; where a warm substep's residual (max |len / rest - 1| over the stretch
           constraints) exceeds that cloth's largest residual under the plain solver over the same
           steps, it keeps iterating (4 at a time, at most 20): equal residual, cloth by cloth.
  roofline shared-memory bound (the cloth lives in shared memory during a step): algorithmic
           bytes per step = sum over cloths of (iterations x constraints x 68 B + particles x
           150 B) x substeps, over the measured per-step duration, against the device's
           shared-memory bandwidth measured on the spot by pxb_measure_smem_bandwidth.
  cpu_baseline  the reference's own solve_cloth (oracle/_ref, compiled from the reference's
           headers, cloths built by the reference's own make_grid_cloth / pin_static /
           build_tethers) on a bounded sample of the workload on this host: 1 thread and all
           threads, at -O2 and at -O3 -march=native.

--impl reference runs only that CPU implementation (rank 0; other ranks exit 0), on this arm's
config, with all host threads; it maps no library of this package.

Several GPUs (torchrun): the batch grows with the ranks (4096 sheets per GPU, weak scaling), is
split over them by cost (physxcoopa_b200/shard.py, largest first onto the least-loaded rank), each
rank steps its share with no collective, and the e2e frames gather every cloth's bounds and speed
to every rank with one all-gather.
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
PLAN_WORKLOADS = ("uneven_batch", "uniform_batch", "single_drape")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["mine", "reference"], default="mine")
    ap.add_argument("--workload", default="uneven_batch",
                    choices=["uneven_batch", "uniform_batch", "single_drape", "warm_start", "hair_groom",
                             "large_cloth_hair", "mesh_floor", "mesh_cloth"])
    ap.add_argument("--cloths", type=int, default=None)
    ap.add_argument("--no-warm", action="store_true",
                    help="uneven batch: leave out the warm-start comparison")
    ap.add_argument("--shear-compliance", type=float, default=None,
                    help="give the shear constraints their own compliance (library extension; the "
                         "reference arm cannot run it)")
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
    ap.add_argument("--cpu-seconds", type=float, default=3.0,
                    help="wall seconds of reference CPU work per timed sample")
    ap.add_argument("--graph", action="store_true",
                    help="step through the captured CUDA graph (pxb_cloths_step_graph) instead of pxb_cloths_step")
    ap.add_argument("--variant", type=int, default=None,
                    help="fix the kernel variant (0/1/2) instead of autotuning")
    ap.add_argument("--launch", choices=["queue", "cta"], default="queue",
                    help="with --variant: persistent work-queue kernels (queue) or one CTA per cloth (cta)")
    ap.add_argument("--iterations", type=int, default=None,
                    help="constraint iterations per substep of the cloth workloads (default: the workload's, 10)")
    ap.add_argument("--thread-fit", type=int, choices=[0, 1], default=None,
                    help="threads per CTA of one-CTA grid sheets: 1 splits an SM between the CTAs its shared "
                         "memory holds, 0 gives each sheet its own count")
    ap.add_argument("--lean-mid", type=int, choices=[0, 1], default=None,
                    help="sheets an SM holds one of when held whole: 1 lean where that holds two or more, 0 whole")
    ap.add_argument("--no-lean-arrays", action="store_true",
                    help="lay sheets of sides 110-128 out on 2-CTA clusters instead of one CTA with float arrays")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------
# workloads
# ------------------------------------------------------------------------------------------

def sheet_params(args):
    from physxcoopa_b200 import scenes
    p = (scenes.reference_params() if args.shear_compliance is None
         else scenes.cloth_params(shear_compliance=args.shear_compliance))
    if args.self_collision:  # at the builder's self_distance (0.6 x spacing)
        p.self_collision = 1
    return p


def total_cloths(args, world):
    """Sheets of the whole job: the configuration's batch per GPU (weak scaling)."""
    default = {"uneven_batch": 4096, "uniform_batch": 1024, "single_drape": 1}[args.workload]
    return (args.cloths or default) * world


def plan(args, world):
    """(name, specs) of a plan workload: every sheet's draws, before any builder runs."""
    from physxcoopa_b200 import scenes
    n = total_cloths(args, world)
    if args.workload == "uneven_batch":
        return scenes.uneven_name(n), scenes.uneven_plan(n, seed=2)
    if args.workload == "uniform_batch":
        return scenes.uniform_name(n, args.side), scenes.uniform_plan(n, args.side, seed=1)
    return scenes.single_drape_name(), scenes.single_drape_plan(seed=0)


def workload_config(args, name, n_cloths, vertices, substeps=4, iterations=10, h=1.0 / 60.0, n_gpus=1):
    """The `config` of the JSON line: identical in both arms for the same arguments."""
    cfg = {"workload": name, "cloths": n_cloths, "vertices": vertices, "substeps": substeps,
           "iterations": iterations, "h": h,
           "compliance": ("structural and shear 0 (ClothParams::stretch_compliance, the reference's one "
                          "stretch compliance), bend 1e-4" if args.shear_compliance is None else
                          f"structural 0 / shear {args.shear_compliance:g} / bend 1e-4 (per-batch compliance)"),
           "l2": "inputs larger than L2 (device state of the batch exceeds 126 MB)"
           if vertices * 64 > 126e6 else "inputs fit in L2",
           "parallelism": f"independent cloths, {n_gpus} GPU(s), cost-balanced shares"}
    if args.workload == "uneven_batch":
        cfg["colliders"] = ("1-3 per sheet from sphere r U(0.2,0.5) / capsule r U(0.1,0.3) half-length "
                            "U(0.2,0.6) / box half-extents U(0.1,0.5), random orientations; half the "
                            "sheets under one point source (9.81, 1 m, 10 m)")
    if args.self_collision:
        cfg["self_collision"] = "on, self_distance 0.6 x spacing"
    return cfg


def build_gpu_scene(args, rank, world):
    """The scene this rank steps. Plan workloads: this rank's cost-balanced share of the job's
    sheets (all of them on one GPU), built by the library's builders."""
    from physxcoopa_b200 import scenes, shard
    if args.workload in PLAN_WORKLOADS:
        name, specs = plan(args, world)
        costs = [shard.cloth_cost(s.side * s.side) for s in specs]
        shares = shard.partition(costs, world)
        mine = shares[rank]
        params = sheet_params(args)
        cloths = [scenes.build_sheet(specs[i], params) for i in mine]
        sc = scenes.ClothScene(name, cloths, [specs[i].colliders for i in mine],
                               sources=[specs[i].source for i in mine])
        return sc, shares, sum(s.side * s.side for s in specs), len(specs)
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
    else:  # mesh_cloth
        sc = scenes.mesh_cloth_batch(n=args.cloths or 1024, rings=args.rings, seed=13 + rank)
    if args.self_collision:
        for c in sc.cloths:
            c.params.self_collision = 1
    return sc, None, sc.vertices * world, len(sc.cloths) * world


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
# the reference CPU implementation (oracle/_ref) on the host cores
# ------------------------------------------------------------------------------------------

CPU_BUILDS = {"O2": ("libpxbref.so", "-O2"), "native": ("libpxbref_native.so", "-O3 -march=native")}


def _ref_handles(lib, specs, params):
    """The sheets built by the reference's own builders: make_grid_cloth (with the seeded jitter),
    pin_static at each pin, build_tethers when pinned."""
    import ctypes as C
    from physxcoopa_b200 import scenes
    hs = []
    for s in specs:
        d = scenes.grid_desc(s.side, s.center, s.seed, params)
        h = lib.pxbref_cloth_make_grid(C.byref(d))
        for point, radius in s.pins:
            lib.pxbref_cloth_pin_static(h, (C.c_float * 3)(*point), radius)
        if s.pins:
            lib.pxbref_cloth_build_tethers(h)
        hs.append(h)
    return hs


def _ref_cpu_child(q, build, plan_args, params_blob, threads, steps, warmup, target_s):
    """Runs in a spawned process (a reference build that does not run on this CPU, or any crash,
    ends only this process). Builds a sample of the plan's sheets with the reference's builders,
    sized so one step over it takes about target_s on `threads` threads, then steps it warmup +
    steps times with pxbref_bench_cloths (the reference's solve_cloth per cloth, whole cloths per
    thread). Puts (rates per timed step, sample size, threads) on q."""
    import ctypes as C
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _checkers as K
    from physxcoopa_b200 import _abi as A
    args = argparse.Namespace(**plan_args)
    _, specs = plan(args, 1)
    params = A.ClothParams.from_buffer_copy(params_blob)
    lib = K.load_ref(os.path.join(ROOT, "oracle", "_ref", CPU_BUILDS[build][0]))
    g = K.vec((0.0, 0.0, -9.81))

    def run(handles, idx, n_steps, nthreads):
        cols = [specs[i].colliders for i in idx]
        flat = np.ascontiguousarray(np.concatenate(cols))
        offs = np.zeros(len(idx) + 1, np.uint32)
        offs[1:] = np.cumsum([len(c) for c in cols])
        srcs = [specs[i].source if specs[i].source is not None else np.zeros(0, A.GRAVITY_SOURCE) for i in idx]
        sflat = np.ascontiguousarray(np.concatenate(srcs)) if srcs else np.zeros(0, A.GRAVITY_SOURCE)
        soffs = np.zeros(len(idx) + 1, np.uint32)
        soffs[1:] = np.cumsum([len(x) for x in srcs])
        hv = (C.c_void_p * len(handles))(*handles)
        return lib.pxbref_bench_cloths(hv, len(handles), A.ptr(flat), A.ptr(offs), A.ptr(sflat), A.ptr(soffs),
                                       g, 4, 10, 1.0 / 60.0, n_steps, nthreads)

    # calibrate on the plan's first sheets, one thread
    probe_idx = list(range(min(8, len(specs))))
    probe = _ref_handles(lib, [specs[i] for i in probe_idx], params)
    wall = run(probe, probe_idx, 1, 1)
    per_vertex = wall / max(1, sum(specs[i].side ** 2 for i in probe_idx))
    for h in probe:
        lib.pxbref_cloth_free(h)
    budget = target_s * threads / max(per_vertex, 1e-12)
    n, acc = 0, 0
    while n < len(specs) and (acc < budget or n < threads):
        acc += specs[n].side ** 2
        n += 1
    idx = list(range(n))
    handles = _ref_handles(lib, [specs[i] for i in idx], params)
    verts = sum(specs[i].side ** 2 for i in idx) * 4
    for _ in range(warmup):
        run(handles, idx, 1, threads)
    rates = [verts / run(handles, idx, 1, threads) for _ in range(steps)]
    for h in handles:
        lib.pxbref_cloth_free(h)
    q.put({"rates": rates, "n_sample": n, "threads": threads})


def ref_cpu(args, build, threads, steps, warmup, target_s):
    """One CPU mode of the reference (build x threads) in a spawned process. Returns the child's
    dict, or {"unavailable": why}."""
    import multiprocessing as mp
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", CPU_BUILDS[build][0])):
        return {"unavailable": f"oracle/_ref/{CPU_BUILDS[build][0]} was not built"}
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    plan_args = {"workload": args.workload, "cloths": args.cloths, "side": args.side}
    p = ctx.Process(target=_ref_cpu_child, args=(q, build, plan_args, bytes(sheet_params(args)), threads, steps,
                                                 warmup, target_s))
    p.start()
    res = None
    deadline = time.time() + 600
    while time.time() < deadline:
        try:
            res = q.get(timeout=1.0)
            break
        except Exception:  # queue.Empty
            if not p.is_alive():
                break
    p.join(timeout=30)
    if res is None:
        return {"unavailable": f"the {CPU_BUILDS[build][1]} build did not run here (exit code {p.exitcode})"}
    return res


def cpu_modes(args, steps=1, warmup=0, target_s=None):
    """The reference on this host: 1 thread and all threads, each at -O2 and -O3 -march=native."""
    target_s = target_s or args.cpu_seconds
    n_all = os.cpu_count() or 1
    modes = {}
    for build in ("O2", "native"):
        for threads in (1, n_all):
            r = ref_cpu(args, build, threads, steps, warmup, target_s)
            key = f"{build}_{threads}thread" if threads == 1 else f"{build}_{threads}threads"
            if "unavailable" in r:
                modes[key] = r
            else:
                modes[key] = {"value": statistics.median(r["rates"]), "flags": CPU_BUILDS[build][1],
                              "threads": threads, "sample_cloths": r["n_sample"], "timed_steps": len(r["rates"])}
    return modes


def cpu_baseline_from_modes(modes, n_total):
    """The all-threads mode of the faster build is the baseline; every mode is listed."""
    best = None
    for k, m in modes.items():
        if "value" in m and m["threads"] > 1 and (best is None or m["value"] > modes[best]["value"]):
            best = k
    if best is None:
        return None
    m = modes[best]
    return {"value": m["value"], "unit": UNIT, "cores": m["threads"], "kind": "reference",
            "sample": f"first {m['sample_cloths']} of {n_total} sheets of the workload, built by the reference's "
                      f"make_grid_cloth / pin_static / build_tethers, stepped by its solve_cloth (serial per cloth, "
                      f"whole cloths over {m['threads']} host threads), {m['flags']}; median of {m['timed_steps']} "
                      f"step(s)",
            "modes": modes}


def reference_arm(args):
    """--impl reference: the reference's solve_cloth on the host cores, on this arm's config."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.workload not in PLAN_WORKLOADS:
        print(json.dumps({"impl": "reference", "unavailable": f"the reference arm runs the sheet workloads "
                                                              f"{', '.join(PLAN_WORKLOADS)}"}))
        return 0
    if args.shear_compliance is not None:
        print(json.dumps({"impl": "reference", "unavailable": "the reference's ClothParams has one stretch "
                                                              "compliance; a separate shear compliance is a "
                                                              "library extension"}))
        return 0
    name, specs = plan(args, world)
    n_all = os.cpu_count() or 1
    W = max(args.warmup, 0)
    target = min(args.cpu_seconds, 180.0 / max(1, args.steps + W))
    per_build = {}
    for build in ("O2", "native"):
        per_build[build] = ref_cpu(args, build, n_all, args.steps, W, target)
    ok = {b: r for b, r in per_build.items() if "rates" in r}
    if not ok:
        print(json.dumps({"impl": "reference", "unavailable": "; ".join(r["unavailable"] for r in per_build.values())}))
        return 0
    best = max(ok, key=lambda b: statistics.median(ok[b]["rates"]))
    value = statistics.median(ok[best]["rates"])
    modes = {}
    for b, r in per_build.items():
        modes[f"{b}_{n_all}threads"] = ({"value": statistics.median(r["rates"]), "flags": CPU_BUILDS[b][1],
                                         "threads": n_all, "sample_cloths": r["n_sample"],
                                         "timed_steps": len(r["rates"])} if "rates" in r else r)
    for b in ("O2", "native"):  # one-thread figures beside them (two samples each)
        r = ref_cpu(args, b, 1, 2, 0, 2.0)
        modes[f"{b}_1thread"] = ({"value": statistics.median(r["rates"]), "flags": CPU_BUILDS[b][1], "threads": 1,
                                  "sample_cloths": r["n_sample"], "timed_steps": len(r["rates"])}
                                 if "rates" in r else r)
    cb = {"value": value, "unit": UNIT, "cores": n_all, "kind": "reference",
          "sample": f"first {ok[best]['n_sample']} of {len(specs)} sheets per step, built by the reference's "
                    f"make_grid_cloth / pin_static / build_tethers and stepped by its solve_cloth (serial per cloth, "
                    f"whole cloths over {n_all} host threads), {CPU_BUILDS[best][1]} (the faster build)",
          "modes": modes}
    vertices = sum(s.side * s.side for s in specs)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": W, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes)",
            "config": workload_config(args, name, len(specs), vertices, n_gpus=world),
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------------------------------
# other workloads
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
    e0 = time.perf_counter()
    for f in range(max(3, args.steps // 2)):
        pos, rot = sc.root_path(f + 1)
        ctx.set_strand_roots(sid, pos, rot)
        ctx.step_strands([sid], [sc.meta["colliders_at"](f + 1)], iterations=sc.iterations)
        ctx.read_strand_particles(sid, n)
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
                    "h2d_bytes_per_step": 200 + 312 + 64 * len(hair.sets[0].strands) + 312,
                    "d2h_bytes_per_step": 12 * n_cloth + 40 * n_hair},
            "roofline": None, "cpu_baseline": None, "gpu_launches": launches, "clocks": clk}
    del keep_c, keep_s
    ctx.close()
    return line


# ------------------------------------------------------------------------------------------
# the learned warm start (config 4) on a cloth batch
# ------------------------------------------------------------------------------------------

def warm_start_comparison(args, ctx, sc, local_rank, steps, tuned=False):
    """Plain 20 iterations against the network + 4 iterations at equal per-cloth residual, on a
    fresh copy of `sc` each run (see the module docstring). Each arm runs at its best kernel
    configuration: the plain arm at the context's autotuned block size and launch form (tuned
    here unless `tuned` or --variant), the warm arm at the faster of its two block sizes (512 and
    1024 threads). Returns a dict for the JSON line."""
    import torch
    from physxcoopa_b200 import scenes
    plain_iters, warm_iters = 20, 4
    if args.variant is not None:
        ctx.set_cloth_variant(args.variant)
        ctx.set_launch_mode(1 if args.launch == "queue" else 0)
    elif not tuned:
        ids = [ctx.add_cloth(c) for c in sc.cloths]
        d, keep = ctx.make_step(ids, sc.colliders, sc.gravity, sc.sources, sc.substeps, plain_iters, sc.h)
        ctx.autotune(d, trials=2)
        for i in ids:
            ctx.remove_cloth(i)
        del keep
    plain_variant = ctx.cloth_variant
    # --- training rows from the plain solver on a separately seeded batch -------------------
    t0 = time.perf_counter()
    tr = scenes.uneven_batch(n=512, seed=102, params=sheet_params(args))
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

    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))
    W = max(args.warmup, 3)

    def run(kind, taus=None, collect=False):
        """Steps a fresh copy of the batch: W plain warm-up steps, then `steps` of `kind`. Timed
        with CUDA events unless `collect`, which reads the per-step warm results instead."""
        ids = [ctx.add_cloth(c) for c in sc.cloths]
        d, keep = ctx.make_step(ids, sc.colliders, sc.gravity, sc.sources, sc.substeps, plain_iters, sc.h)
        for _ in range(W):
            ctx.step_desc(d)
        ctx.synchronize()
        res = []
        t_a, t_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launch_count
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            t_a.record(stream)
            for _ in range(steps):
                if kind == "plain":
                    ctx.step_desc(d)
                elif kind == "plain_residual":
                    ctx.step_warm_desc(d, warm_iterations=0)
                elif kind == "warm_restart":
                    ctx.step_warm_desc(d, warm_iterations=warm_iters, thresholds=taus)
                else:
                    ctx.step_warm_desc(d, warm_iterations=warm_iters, thresholds=taus, continue_iterations=True)
                if collect:
                    res.append(ctx.read_warm_results(ids))
            t_b.record(stream)
        torch.cuda.synchronize()
        ms = t_a.elapsed_time(t_b) / steps
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
    subs = sum(r["substeps"].sum() for r in res_w)
    fb = float(sum(r["fallbacks"].sum() for r in res_w) / subs)
    extra = float(sum(r["extra_iterations"].sum() for r in res_w) / subs)
    # the warm kernel comes in two block sizes (variants 0 and 1-2 run 512 and 1024 threads)
    warm_ms = {}
    for v in ((args.variant,) if args.variant is not None else (0, 2)):
        ctx.set_cloth_variant(v)
        warm_ms[v] = run("warm", taus)
    best_v = min(warm_ms, key=lambda v: warm_ms[v][0])
    ms_warm, _, launches = warm_ms[best_v]
    ctx.set_cloth_variant(best_v)
    ms_restart, _, _ = run("warm_restart", taus)
    ctx.set_cloth_variant(plain_variant)
    verts = sc.vertices * sc.substeps
    return {"workload": "the same batch: 20 plain iterations vs the network + 4 iterations, equal residual "
                        "cloth by cloth",
            "plain": {"iterations": plain_iters, "value": verts / (ms_plain * 1e-3), "ms_per_step": ms_plain,
                      "residual_median": float(np.median(rp)), "residual_max": float(rp.max())},
            "warm": {"iterations": warm_iters, "value": verts / (ms_warm * 1e-3), "ms_per_step": ms_warm,
                     "residual_median": float(np.median(rw)), "residual_max": float(rw.max()),
                     "gpu_launches": launches},
            "speedup_vs_plain": ms_plain / ms_warm,
            "kernels": {"plain_block_cap": [512, 768, 1024][plain_variant],
                        "warm_block_threads": {[512, 1024, 1024][v]: warm_ms[v][0] for v in warm_ms},
                        "launch": "persistent work queue" if ctx.launch_mode == 1 else "one CTA per cloth"},
            "fallback_rate": fb, "extra_iterations_per_substep": extra,
            "fallback": "continue iterating from the warm state, 4 at a time, to the threshold or 20 iterations",
            "restart_fallback": {"ms_per_step": ms_restart, "speedup_vs_plain": ms_plain / ms_restart,
                                 "note": "restart from the prediction with 20 plain iterations"},
            "residual": "max |len/rest - 1| over the stretch constraints, per cloth and substep",
            "equal_residual": "a warm substep keeps iterating while its residual exceeds the plain solver's largest "
                              "residual for that cloth over the same steps",
            "dtype": "f32 solve; network bf16 weights and activations, fp32 accumulation (tcgen05, TMEM)",
            "timed_steps": steps,
            "training": {"rows": int(len(X)), "final_loss": loss, "record_s": t_rec, "train_s": t_train,
                         "scenes": f"uneven batch seed 102 (512 sheets), plain 20 iterations, {rec_steps} steps"}}


def bench_warm(args, local_rank):
    """--workload warm_start: the comparison alone on the uneven batch, as its own JSON line."""
    from physxcoopa_b200 import runtime as R
    from physxcoopa_b200 import scenes
    ctx = R.Context(local_rank)
    sc = scenes.uneven_batch(n=args.cloths or 4096, seed=2, params=sheet_params(args))
    clocks = ClockSampler(local_rank)
    clocks.start()
    w = warm_start_comparison(args, ctx, sc, local_rank, args.steps)
    clk = clocks.stop()
    ctx.close()
    return {"metric": METRIC, "value": w["warm"]["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": w["warm"]["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 solve, bf16 network (fp32 accumulation)",
            "data": "synthetic (seeded scenes)",
            "config": dict(workload=f"warm_start on {sc.name}", cloths=len(sc.cloths), vertices=sc.vertices),
            "warm_start": w, "roofline": None, "cpu_baseline": None, "gpu_launches": w["warm"]["gpu_launches"],
            "clocks": clk}


# ------------------------------------------------------------------------------------------
# main: a cloth batch
# ------------------------------------------------------------------------------------------

def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        return reference_arm(args)

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
    from physxcoopa_b200 import shard

    sc, shares, job_vertices, job_cloths = build_gpu_scene(args, rank, world)
    if args.iterations:
        sc.iterations = args.iterations
    ctx = R.Context(local_rank)
    if args.no_lean_arrays:
        ctx.set_lean_arrays(False)
    if args.thread_fit is not None:
        ctx.set_thread_fit(args.thread_fit)
    if args.lean_mid is not None:
        ctx.set_lean_mid(args.lean_mid)
    if sc.geometries:
        from physxcoopa_b200 import scenes
        scenes.register_geometries(ctx, sc)
    ids = [ctx.add_cloth(c) for c in sc.cloths]
    d, keep = ctx.make_step(ids, sc.colliders, sc.gravity, sc.sources, sc.substeps,
                            sc.iterations, sc.h)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local_rank))

    if args.variant is None:
        best, ms = ctx.autotune(d, trials=2)
        tune = {"chosen": {"block_cap": [512, 768, 1024][best % 3],
                           "launch": "persistent work queue" if best >= 3 else "one CTA per cloth"},
                "ms_per_step": {"one CTA per cloth": ms[:3], "persistent work queue": ms[3:]},
                "variants": "block-size cap 512 / 768 / 1024 threads x launch form, then per layout class",
                "thread_fit": ctx.tuning()["thread_fit"],
                "classes": ctx.tuning()["classes"]}
    else:
        ctx.set_cloth_variant(args.variant)
        ctx.set_launch_mode(1 if args.launch == "queue" else 0)
        tune = {"chosen": {"block_cap": [512, 768, 1024][args.variant],
                           "launch": "persistent work queue" if args.launch == "queue" else "one CTA per cloth"},
                "fixed": True}
    step = ctx.step_graph_desc if args.graph else ctx.step_desc
    W = max(args.warmup, 3)
    for _ in range(W):
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

    value = job_vertices * sc.substeps * args.steps / (elapsed_ms * 1e-3)

    # --- roofline of the dominant kernel (shared memory), this rank's share ------------------
    cons = sum(len(c.stretch) + len(c.bend) for c in sc.cloths)
    algo_bytes = sc.substeps * (sc.iterations * cons * 68 + sc.vertices * 150)
    achieved = algo_bytes / (per_launch_ms * 1e-3) / 1e9
    peak = smem_bw / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"cloth_step_{args.workload}.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch_full_workload")
        except (OSError, ValueError):
            traffic = None

    # --- end to end through the public API with host buffers -----------------------------
    e2e_steps = args.e2e_steps or max(3, args.steps // 2)
    from physxcoopa_b200 import _abi as A
    outs_np = [torch.empty(3 * sc.vertices, dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    ids_np = np.ascontiguousarray(ids, np.uint64)
    res_out = np.zeros(len(ids), A.FRAME_RESULT)
    # per-cloth results (bounds, largest speed, time: 32 B per cloth), pinned
    res_pinned = [torch.empty(8 * len(ids), dtype=torch.float32, pin_memory=True).numpy().view(A.FRAME_RESULT)
                  for _ in range(2)]
    # pxb_cloths_step uploads one staging block per step: per-cloth step records (200 B),
    # collider snapshots (312 B), gravity sources (24 B), the launch order (4 B), the launch
    # groups' work-queue counters (4 B per cloth at most) and the posed
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
    h2d = (al(200 * len(ids)) + al(312 * max(n_col, 1)) + al(24 * max(n_src, 1)) + al(4 * len(ids))
           + al(4 * len(ids)) + al(hull_bytes))
    d2h = 12 * sc.vertices + 32 * len(ids) + 4
    ctx.synchronize()

    def timed_e2e(pipelined):
        """Per step: the step call (its inputs uploaded from pinned memory), every particle
        position and the per-cloth results read back to pinned host memory. Pipelined:
        pxb_cloths_read_positions_async / pxb_cloths_read_results_async, step k's read-back
        copied while step k + 1 is prepared and runs, every copy landed before the closing
        event; else the blocking pxb_cloths_read_positions / pxb_cloths_read_results. With
        several ranks each frame's results are gathered to every rank (one all-gather)."""
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
                    if dist:  # the broadphase of every rank needs this frame's results
                        ctx.wait_positions()
                        shard.gather_results(res_pinned[k % 2], shares, job_cloths)
                else:
                    ctx.read_positions(ids_np, outs_np[0])
                    ctx.lib.pxb_cloths_read_results(ctx.h, A.ptr(ids_np), len(ids_np), A.ptr(res_out))
                    if dist:
                        shard.gather_results(res_out, shares, job_cloths)
            if pipelined:
                ctx.wait_positions()
            e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t[0])
        return job_vertices * sc.substeps * e2e_steps / (ms * 1e-3)

    e2e_blocking = timed_e2e(False)
    e2e_value = timed_e2e(True)

    # --- the learned warm start on the same batch (rank 0, one GPU) -------------------------
    warm = None
    if args.workload == "uneven_batch" and not args.no_warm and rank == 0 and world == 1:
        warm = warm_start_comparison(args, ctx, sc, local_rank, args.steps, tuned=True)

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline and args.workload in PLAN_WORKLOADS:
            cpu = cpu_baseline_from_modes(cpu_modes(args), job_cloths)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": W, "ms_per_step": elapsed_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scenes)",
            "config": workload_config(args, sc.name, job_cloths, job_vertices, sc.substeps, sc.iterations, sc.h,
                                      n_gpus=world),
            "launch": {"entry": "pxb_cloths_step_graph (captured CUDA graph)" if args.graph else "pxb_cloths_step",
                       "autotune": tune,
                       "sides_110_128": "two-CTA clusters" if args.no_lean_arrays else "one CTA, positions as float arrays"},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "read_back": "pipelined: pxb_cloths_read_positions_async + pxb_cloths_read_results_async, "
                                 "each step's positions and results copied to pinned host memory while the "
                                 "next step is prepared and runs",
                    "blocking_value": e2e_blocking},
            "warm_start": warm,
            "roofline": {"bound": "smem", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "measured on this GPU by pxb_measure_smem_bandwidth",
                         "kernel": "cloth_step_kernel", "per_launch_ms": per_launch_ms,
                         "per_launch": "one pxb_cloths_step (all of the step's grouped launches)",
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "hbm": hbm_roofline(traffic, per_launch_ms)},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk,
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
