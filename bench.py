#!/usr/bin/env python
"""Throughput of the plain rigid-body step (body-substeps per second) on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl natsel|reference]

Workload (default): the 10 000-body pile, i.e. 6 000 boxes, 2 500 spheres and 1 500 capsules
dropped from a 40 x 60 x 40 m volume onto a ground box, stepped at 60 Hz with 4 substeps in
FP32 (scene builder ``natsel_b200.scenes.large_pile``; seeded synthetic data). A step is one
``World::step`` (solver_integration.rs:807 in the reference): broadphase pair update,
narrowphase, colouring, prepare, the substep solve and finalize. The timed steps are
W+1 .. W+K of the drop.

natsel arm (default): one world per GPU (replicas, weak scaling; no collective on the data
path). ``value`` is the device time of the K steps measured with CUDA events on the world's
stream, with the L2 flushed between steps outside the events (the working set fits in L2);
``e2e`` repeats the run through the public C ABI with per-step host inputs (external forces,
copied host->device) and the full body state read back to pinned host memory every step.
``roofline`` is for the persistent solver kernel (k_solve): algorithmic bytes per launch from
the per-step solver counts divided by its CUDA-event duration. ``cpu_baseline`` times the CPU
oracle (a scalar C++ restatement of the reference step) on a bounded sample of the same drop.

reference arm (``--impl reference``): the reference engine is Rust and cannot be built on
this image, so its CPU step is timed through the oracle port on a bounded sample of the same
workload: one world colour-parallel on every host core, as the reference parallelises a world
(``--reference-mode replicas``: one replica world per core instead; batched worlds always run
one world per core); under torchrun only rank 0 runs it.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 1.0 / 60.0
FLUSH_BYTES = 256 << 20  # > 126 MB L2
METRIC = "body-substeps/s"

WORKLOADS = {
    "large_pile": ("large_pile", {}, "10 000 dynamic bodies (6 000 boxes h U(0.25,0.75), 2 500 spheres r U(0.2,0.6), "
                                     "1 500 capsules r U(0.15,0.4) hh U(0.2,0.8)) dropped from a 40x60x40 m volume "
                                     "onto a ground box; 60 Hz, 4 substeps, FP32"),
    "box_pyramid": ("box_pyramid", {}, "pyramid of 210 unit cubes (base 20) on a ground box; 60 Hz, 4 substeps, FP32"),
    "large_pyramid": ("large_pyramid", {}, "the reference's large_pyramid benchmark scene (5 050 boxes resting from the "
                                           "first step, scenes.rs:105); 60 Hz, 4 substeps, FP32"),
    "batched_worlds": ("batched_worlds", {"count": 4096, "seed": 4},
                       "4 096 independent worlds, each a box pyramid or a random drop (shape mix and ranges of the "
                       "10 000-body pile) of N ~ log-uniform(32, 512) bodies, stepped together; 60 Hz, 4 substeps, FP32"),
    "jointed_chains": ("jointed_chains", {}, "2 000 chains of 24 capsules on limited revolute joints + 4 000 boxes; "
                                             "60 Hz, 8 substeps, FP32"),
    "differentiable_rollout": ("differentiable_rollout", {},
                               "1 024 unit cubes on a ground box with v0 ~ N(0, 2^2) m/s and w0 ~ N(0, 1) rad/s, "
                               "64 steps at 60 Hz with 4 substeps, loss sum |x_final - x_target|^2, gradients "
                               "w.r.t. initial velocities, masses and frictions by the adjoint (ns_world_vjp) "
                               "with checkpoints every 8 substeps; FP32"),
}
ROLLOUT_CHECKPOINT = 8


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=3, help=">= 1 (the first step uploads the scene)")
    ap.add_argument("--impl", choices=["natsel", "reference"], default="natsel")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="large_pile")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--reference-seconds", type=float, default=60.0, help="budget of the reference arm's timed sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-mode", choices=["colour-parallel", "replicas"], default="colour-parallel",
                    help="reference arm for a single world: the oracle colour-parallel on every host core "
                         "(as the reference runs one world), or one replica world per core")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--rollout-steps", type=int, default=64,
                    help="steps of each differentiable rollout (64 in the workload; fewer for profiling)")
    return ap.parse_args(argv)


# ---------------------------------------------------------------------------------------------
# algorithmic bytes of one k_solve launch (the solver stages of one step, all substeps)

def solve_launch_bytes(counts, substeps, restitution_iterations=2):
    """Bytes the solver stages must move for one step, compact FP32 SoA accounting:
    per awake body and substep 116 B integrate-velocity (+40 B when gyroscopic) and 104 B
    integrate-position; per manifold and substep with P points 756 + 120 P B over warm start,
    push and relax, minus 200 B per static side (its body is never read or written); per
    revolute joint and substep 680 B; once per step the impulse store (40 + 16 P B per
    manifold) and, when any contact has restitution, that many push-like passes
    (220 + 40 P B per manifold, minus 76 B per static side)."""
    c = [int(x) for x in counts]
    n_awake, manifolds, points, static_sides, joints = c[0], c[2], c[3], c[4], c[5]
    overflow, gyro, o_points, o_static = c[6], c[8], c[9], c[10]
    m_all, p_all, s_all = manifolds + overflow, points + o_points, static_sides + o_static
    per_substep = n_awake * (116 + 104) + 40 * gyro + 756 * m_all + 120 * p_all - 200 * s_all + 680 * joints
    per_step = 40 * m_all + 16 * p_all
    if c[7]:
        per_step += restitution_iterations * (220 * m_all + 40 * p_all - 76 * s_all)
    return substeps * per_substep + per_step


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(algorithmic_bytes):
    """DRAM bytes per k_solve launch from the committed ncu capture (profiles/k_solve_large_pyramid.md,
    a smaller contact-rich case), scaled to this run by algorithmic bytes; None without it."""
    path = os.path.join(ROOT, "profiles", "k_solve_large_pyramid.md")
    found = {}
    try:
        for line in open(path):
            key, _, val = line.partition(":")
            if key.strip() in ("traffic_bytes_per_launch", "algorithmic_bytes_per_launch") and val.strip():
                found[key.strip()] = float(val.split()[0])
    except OSError:
        return None
    if len(found) < 2 or found["algorithmic_bytes_per_launch"] <= 0:
        return None
    return found["traffic_bytes_per_launch"] / found["algorithmic_bytes_per_launch"] * algorithmic_bytes


# ---------------------------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    QUERY = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, uuids):
        self.uuids = [u.lower().replace("gpu-", "") for u in uuids]
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.seek(0)
        sm, smax, reasons, power = [], [], set(), []
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            uuid = parts[0].lower().replace("gpu-", "")
            if self.uuids and uuid not in self.uuids:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for name, val in zip(self.REASONS, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        self.file.close()
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------------------------
# CPU side (oracle): single-thread baseline and the reference arm's replica workers

def oracle_run(scene, kw, warmup, max_steps, budget_s, barrier=None, first_world=0, world_step=1):
    """Time the oracle on the workload. A batch of worlds is timed world by world (the oracle is
    one world): worlds first_world, first_world + world_step, ... each run warmup + max_steps
    steps, until the budget is spent."""
    from natsel_b200 import scenes
    from oracle import pyoracle
    sub = scenes.SUBSTEPS[scene]
    if scene == "batched_worlds":
        if barrier is not None:
            barrier.wait()
        units, seconds, steps, k = 0, 0.0, 0, first_world
        while seconds < budget_s and k < kw["count"]:
            w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[scene])
            info = scenes.batch_world(w, k, kw["seed"])
            for _ in range(warmup):
                w.step(DT, sub)
            t0 = time.perf_counter()
            for _ in range(max_steps):
                w.step(DT, sub)
            seconds += time.perf_counter() - t0
            units += info["dynamic_bodies"] * sub * max_steps
            steps += max_steps
            k += world_step
        return {"steps": steps, "seconds": seconds, "bodies": units / max(steps, 1) / sub, "substeps": sub,
                "worlds": (k - first_world) // world_step}
    w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[scene])
    info = scenes.BUILDERS[scene](w, **kw)
    for _ in range(warmup):
        w.step(DT, sub)
    if barrier is not None:
        barrier.wait()
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps:
        w.step(DT, sub)
        steps += 1
        if time.perf_counter() - t0 > budget_s:
            break
    return {"steps": steps, "seconds": time.perf_counter() - t0, "bodies": info["dynamic_bodies"], "substeps": sub}


def _replica_worker(scene, kw, warmup, max_steps, budget_s, barrier, queue, first_world=0, world_step=1):
    try:
        queue.put(oracle_run(scene, kw, warmup, max_steps, budget_s, barrier, first_world, world_step))
    except Exception as e:  # report instead of hanging the parent
        queue.put({"error": repr(e)})


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference_arm(args):
    import multiprocessing as mp
    from oracle import pyoracle
    pyoracle.build()
    scene, kw, desc = WORKLOADS[args.workload]
    n = min(host_cores(), 128)
    if scene != "batched_worlds" and args.reference_mode == "colour-parallel":
        return run_reference_colour_parallel(args, scene, kw, desc, n)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(n)
    queue = ctx.Queue()
    procs = [ctx.Process(target=_replica_worker, args=(scene, kw, args.warmup, args.steps, args.reference_seconds,
                                                        barrier, queue, r, n)) for r in range(n)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=args.reference_seconds + 600) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    errors = [r["error"] for r in results if "error" in r]
    if errors:
        raise RuntimeError("reference replica failed: %s" % errors[0])
    seconds = max(r["seconds"] for r in results)
    units = sum(r["steps"] * r["bodies"] * r["substeps"] for r in results)
    value = units / seconds
    steps = min(r["steps"] for r in results)
    ms_per_step = 1000.0 * statistics.mean(r["seconds"] / r["steps"] for r in results)
    if scene == "batched_worlds":
        sample = ("%d processes (one per host core, %s) stepping the batch's worlds one after another, "
                  "%d worlds, steps %d..%d of each (bounded to %.0f s)" % (
                      n, cpu_model(), sum(r.get("worlds", 0) for r in results), args.warmup + 1,
                      args.warmup + args.steps, args.reference_seconds))
    else:
        sample = ("%d replica worlds (one per host core, %s), each timing steps %d..%d of the drop "
                  "(bounded to %.0f s)" % (n, cpu_model(), args.warmup + 1, args.warmup + steps, args.reference_seconds))
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene builder, no dataset)",
        "config": config_block(args, desc), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_steps_per_replica": steps,
    }
    print(json.dumps(line), flush=True)


def run_reference_colour_parallel(args, scene, kw, desc, n):
    """One world, as the reference steps it: the oracle's colour-parallel loops (collide per
    contact, prepare and every solver stage per constraint of a colour, the body stages per body;
    the pair update, the ordered state pass and the overflow colour stay serial) on every host
    core, timing steps W+1..W+K of the workload within the time budget."""
    from oracle import pyoracle
    pyoracle.set_threads(n)
    r = oracle_run(scene, kw, args.warmup, args.steps, args.reference_seconds)
    pyoracle.set_threads(1)
    value = r["steps"] * r["bodies"] * r["substeps"] / r["seconds"]
    sample = ("one world, colour-parallel on %d host threads (%s), steps %d..%d (bounded to %.0f s)" % (
        n, cpu_model(), args.warmup + 1, args.warmup + r["steps"], args.reference_seconds))
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * r["seconds"] / r["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene builder, no dataset)",
        "config": config_block(args, desc), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_steps": r["steps"],
    }
    print(json.dumps(line), flush=True)


def config_block(args, desc):
    return {"workload": "%s: %s" % (args.workload, desc), "first_timed_step": args.warmup + 1,
            "timed_steps": args.steps, "l2": "flushed between steps (256 MiB write outside the timed events)",
            "parallelism": "replicas: one independent world per GPU (%d)" % args.gpus}


# ---------------------------------------------------------------------------------------------
# natsel arm

def build_gpu_world(args, device):
    from natsel_b200 import scenes
    from natsel_b200.world import World, default_world_def
    scene, kw, _ = WORKLOADS[args.workload]
    s = scenes.WORLD_SETTINGS[scene]
    w = World(default_world_def(gravity=s["gravity"], enable_continuous=int(s["enable_continuous"]), device=device))
    info = scenes.BUILDERS[scene](w, **kw)
    return w, info, scenes.SUBSTEPS[scene]


def make_reducer(world_size, device):
    """reduce(x, "max" | "sum") over the ranks of the default process group (identity alone)."""
    import torch
    import torch.distributed as dist

    def reduce(x, op):
        if world_size == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return float(t.item())
    return reduce


def job_throughput(bodies, substeps, steps, elapsed_ms, reduce):
    """Whole-job body-substeps/s: the bodies of every rank over the slowest rank's time.
    Returns (value, max elapsed ms)."""
    total_ms = reduce(float(elapsed_ms), "max")
    units = reduce(float(bodies), "sum") * substeps * steps
    return units / (total_ms / 1000.0), total_ms


def run_natsel_arm(args):
    import numpy as np
    import torch
    import torch.distributed as dist
    from natsel_b200 import _build

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("bench.py: the natsel arm needs a CUDA device")
    if not os.path.exists(_build.LIB):
        raise SystemExit("bench.py: libnatsel_gpu.so is missing; run __graft_entry__.build()")
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world_size > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world_size > 1:
            dist.barrier()
        torch.cuda.synchronize()

    reduce = make_reducer(world_size, dev)

    uuids = [str(torch.cuda.get_device_properties(local_rank).uuid)]
    if world_size > 1:
        gathered = [None] * world_size
        dist.all_gather_object(gathered, uuids[0])
        uuids = gathered

    scene, kw, desc = WORKLOADS[args.workload]
    if scene == "differentiable_rollout":
        run_rollout_arm(args, rank, local_rank, world_size, dev, barrier, reduce, uuids, desc)
        if world_size > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    world, info, sub = build_gpu_world(args, local_rank)
    bodies = info["dynamic_bodies"]
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        world.step(DT, sub)
    world.synchronize()
    autotune = None
    if scene == "batched_worlds":
        # the solver's launch shape for this batch, timed from a copy of its state (unchanged)
        autotune = [{"blocks": b, "cooperative_grid": g, "ms_per_step": ms} for b, g, ms in world.autotune(DT, sub, 3)]
    stream = torch.cuda.ExternalStream(world.stream(), device=dev)  # created by the first step
    launches0 = int(world.solver_counts()[12])

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    phase = np.zeros((args.steps, 5), np.float64)
    solve_bytes = np.zeros(args.steps, np.float64)
    barrier()
    sampler = ClockSampler(uuids) if rank == 0 else None
    wall0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush.zero_()
            starts[k].record(stream)
            world.step(DT, sub)
            ends[k].record(stream)
            ends[k].synchronize()
            phase[k] = world.phase_times()
            solve_bytes[k] = solve_launch_bytes(world.solver_counts(), sub)
    world.synchronize()
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop() if sampler else None
    launches = int(world.solver_counts()[12]) - launches0
    step_ms = np.array([s.elapsed_time(e) for s, e in zip(starts, ends)])
    value, total_ms = job_throughput(bodies, sub, args.steps, float(step_ms.sum()), reduce)
    launches = int(reduce(float(launches), "sum"))

    solve_ms = phase[:, 3]
    achieved = solve_bytes.sum() / (solve_ms.sum() / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    traffic = profiled_traffic(float(solve_bytes.mean()))
    roofline = {"kernel": "k_solve", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic,
                "traffic_source": "ncu capture of k_solve on large_pyramid (profiles/), scaled by algorithmic bytes",
                "algorithmic_bytes_per_launch": float(solve_bytes.mean()),
                "launch_ms": float(solve_ms.mean())}

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, local_rank, dev, barrier, reduce, world_size)

    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        r = oracle_run(scene, kw, args.warmup, args.steps, args.cpu_seconds)
        what = ("%d of the batch's worlds one after another, steps %d..%d of each" % (
            r.get("worlds", 0), args.warmup + 1, args.warmup + args.steps)) if scene == "batched_worlds" else (
            "steps %d..%d of the same drop" % (args.warmup + 1, args.warmup + r["steps"]))
        cpu = {"value": r["steps"] * r["bodies"] * r["substeps"] / r["seconds"], "unit": METRIC, "cores": 1,
               "kind": "port",
               "sample": "CPU oracle (scalar C++ restatement of the reference step, 1 thread, %s) timing %s "
                         "(bounded to %.0f s)" % (cpu_model(), what, args.cpu_seconds)}
    one_at_a_time = None
    if rank == 0 and scene == "batched_worlds":
        one_at_a_time = run_one_world_at_a_time(args, local_rank, kw)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene builder, no dataset)", "config": config_block(args, desc),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "gpu_launches": launches,
            "one_world_at_a_time": one_at_a_time,
            "solver_autotune": autotune,
            "wall_s": wall,
            "phase_ms_mean": {k: float(v) for k, v in zip(["broadphase", "collide", "state_color_prepare", "solve",
                                                          "finalize"], phase.mean(0))},
        }
        print(json.dumps(line), flush=True)
    world.close()
    if world_size > 1:
        dist.barrier()
        dist.destroy_process_group()


def rollout_fd_check(args, local_rank, g, n_entries=12, seed=11):
    """Central differences of the rollout's loss for a seeded sample of gradient entries
    (initial velocity components, masses, frictions), each at h and 2 h; entries whose two
    differences agree to 0.2 % are compared with the adjoint (the rest straddle a contact
    kink: a clamp, a corner unloading or a contact beginning inside the interval)."""
    import numpy as np
    from natsel_b200 import scenes
    from natsel_b200.world import World, default_world_def
    s = scenes.WORLD_SETTINGS["differentiable_rollout"]

    def loss(what, body, comp, delta):
        w = World(default_world_def(gravity=s["gravity"], enable_continuous=0, device=local_rank))
        info = scenes.differentiable_rollout(w, perturb=(what, body, comp, delta))
        for _ in range(args.rollout_steps):
            w.step(DT, 4)
        pos = w.bodies()[0][1:]
        w.close()
        return float(np.sum((pos - info["targets"]) ** 2)), info["perturbed_value"]

    rng = np.random.Generator(np.random.PCG64(seed))
    rows = []
    for e in range(n_entries):
        body = int(rng.integers(0, 1024))
        kind = ("velocity", "velocity", "mass", "friction")[e % 4]
        comp = int(rng.integers(0, 3))
        if kind == "velocity":
            what, hs, adj = "v0", 1e-3, float(g["lin0"][body + 1, comp])
        elif kind == "mass":
            # a unit cube: mass = density * 1 m^3, so d/d(density) = d/d(mass)
            what, hs, adj, comp = "density", 1.0, float(g["mass"][body + 1]), 0
        else:
            what, hs, adj, comp = "friction", 1e-3, float(g["friction"][body + 1]), 0
        fds = []
        for h in (hs, 2 * hs):
            lu, vu = loss(what, body, comp, h)
            ld, vd = loss(what, body, comp, -h)
            fds.append((lu - ld) / (vu - vd))
        rows.append({"entry": kind, "body": body, "component": comp, "adjoint": adj, "fd_h": fds[0],
                     "fd_2h": fds[1]})
    clean = [r for r in rows if abs(r["fd_h"] - r["fd_2h"]) <= 2e-3 * abs(r["fd_h"]) and r["fd_h"] != 0.0]
    rel = [abs(r["adjoint"] - r["fd_h"]) / abs(r["fd_h"]) for r in clean]
    return {"entries": len(rows), "smooth_entries": len(clean),
            "max_rel_err_smooth": max(rel) if rel else None,
            "median_rel_err_smooth": statistics.median(rel) if rel else None,
            "within_1e-3_plus_spread": sum(1 for r in clean if abs(r["adjoint"] - r["fd_h"]) <= 1e-3 * abs(r["fd_h"]) +
                                           2 * abs(r["fd_h"] - r["fd_2h"])),
            "rows": rows}


def run_rollout_arm(args, rank, local_rank, world_size, dev, barrier, reduce, uuids, desc):
    """The differentiable rollout: per timed repetition, the plain forward rollout (64 steps, no
    tape), the same rollout recorded on a tape (checkpoint copies every 8 substeps) and its
    vector-Jacobian product, each timed with CUDA events on the world's stream. The headline
    value is body-substeps/s through the recorded forward plus the adjoint; the adjoint's cost
    is reported against the plain forward's."""
    import numpy as np
    import torch
    from natsel_b200 import scenes
    from natsel_b200.world import World, default_world_def
    s = scenes.WORLD_SETTINGS["differentiable_rollout"]

    def fresh():
        w = World(default_world_def(gravity=s["gravity"], enable_continuous=0, device=local_rank))
        info = scenes.differentiable_rollout(w)
        return w, info

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    plain_ms, taped_ms, vjp_ms, e2e_ms, launches = [], [], [], [], []
    f64_check = None
    phase = np.zeros(5)
    sampler = None
    grads = None
    for rep in range(args.warmup + args.steps):
        timed = rep >= args.warmup
        if timed and sampler is None and rank == 0:
            barrier()
            sampler = ClockSampler(uuids)
        # plain forward: one untimed step uploads the scene, then 64 timed steps
        w, info = fresh()
        w.step(DT, 4)
        w.synchronize()
        st = torch.cuda.ExternalStream(w.stream(), device=dev)
        c0 = int(w.solver_counts()[12])
        e0, e1 = events()
        e0.record(st)
        ph = np.zeros(5)
        for _ in range(args.rollout_steps):
            w.step(DT, 4)
        e1.record(st)
        e1.synchronize()
        ph += w.phase_times()
        fwd_launches = int(w.solver_counts()[12]) - c0
        w.close()
        # recorded forward and its adjoint (tape_begin uploads the scene and takes checkpoint 0)
        w, info = fresh()
        w.tape_begin(ROLLOUT_CHECKPOINT)
        w.synchronize()
        st = torch.cuda.ExternalStream(w.stream(), device=dev)
        t0, t1 = events()
        a0, a1 = events()
        wall0 = time.perf_counter()
        t0.record(st)
        for _ in range(args.rollout_steps):
            w.step(DT, 4)
        t1.record(st)
        pos = w.bodies()[0]
        dpos = np.zeros_like(pos, dtype=np.float32)
        dpos[1:] = 2.0 * (pos[1:] - info["targets"])
        a0.record(st)
        g = w.vjp(dpos=dpos)
        a1.record(st)
        a1.synchronize()
        wall = time.perf_counter() - wall0
        tinfo = w.tape_info()
        if tinfo[2]:
            raise SystemExit("bench.py: the adjoint's narrowphase replay missed %d manifolds" % tinfo[2])
        if timed and rep == args.warmup + args.steps - 1 and rank == 0 and not args.no_cpu_baseline:
            h0 = time.perf_counter()
            g64 = w.vjp_f64(dpos=dpos)
            f64_check = {"host_seconds": time.perf_counter() - h0}
            for key in ("lin0", "ang0", "mass", "friction"):
                a_, b_ = np.asarray(g[key], np.float64).ravel(), np.asarray(g64[key]).ravel()
                rel = np.abs(a_ - b_) / np.maximum(np.abs(b_), 1e-3 * np.abs(b_).max() + 1e-300)
                f64_check[key] = {"median_rel": float(np.median(rel)), "p99_rel": float(np.quantile(rel, 0.99)),
                                  "max_rel": float(rel.max()), "frac_within_1e-3": float(np.mean(rel < 1e-3))}
        w.close()
        if timed:
            plain_ms.append(e0.elapsed_time(e1))
            taped_ms.append(t0.elapsed_time(t1))
            vjp_ms.append(a0.elapsed_time(a1))
            e2e_ms.append(1000.0 * wall)
            launches.append(fwd_launches + int(tinfo[6]))
            phase += ph
            grads = g
    clocks = sampler.stop() if sampler else None
    n = 1024
    units = n * 4 * args.rollout_steps
    k = len(plain_ms)
    plain = reduce(float(np.mean(plain_ms)), "max")
    taped = reduce(float(np.mean(taped_ms)), "max")
    vjp = reduce(float(np.mean(vjp_ms)), "max")
    e2e = reduce(float(np.mean(e2e_ms)), "max")
    value = world_size * units / ((taped + vjp) / 1000.0)
    fd = rollout_fd_check(args, local_rank, grads) if (rank == 0 and not args.no_cpu_baseline) else None
    cpu = None
    if rank == 0 and world_size == 1 and not args.no_cpu_baseline:
        r = oracle_run("differentiable_rollout", {}, 1, args.rollout_steps, args.cpu_seconds)
        cpu = {"value": r["steps"] * r["bodies"] * r["substeps"] / r["seconds"], "unit": METRIC, "cores": 1,
               "kind": "port",
               "sample": "CPU oracle forward rollout only (the reference has no adjoint), %d steps, 1 thread, %s"
                         % (r["steps"], cpu_model())}
    solve_ms = phase[3] / max(k, 1) / args.rollout_steps
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (taped + vjp) / args.rollout_steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene builder, no dataset)",
            "config": {"workload": "%s: %s" % (args.workload, desc),
                       "timed_steps": "%d rollouts of %d steps" % (args.steps, args.rollout_steps),
                       "l2": "working set (~40 MB of world and tape) stays in L2 between rollouts; not flushed",
                       "parallelism": "replicas: one independent world per GPU (%d)" % args.gpus},
            "adjoint": {"forward_ms_per_step": plain / args.rollout_steps,
                        "recorded_forward_ms_per_step": taped / args.rollout_steps,
                        "adjoint_ms_per_step": vjp / args.rollout_steps,
                        "adjoint_over_forward": vjp / plain,
                        "recorded_forward_plus_adjoint_over_forward": (taped + vjp) / plain,
                        "checkpoint_substeps": ROLLOUT_CHECKPOINT,
                        "f64_host_adjoint_check": f64_check,
                        "fd_check": fd},
            "roofline": {"kernel": "k_solve (forward rollout)", "bound": "hbm", "achieved": None,
                         "peak": measured_peak()[0], "unit": "GB/s", "frac": None, "traffic": None,
                         "launch_ms": solve_ms,
                         "note": "this workload is measured for the adjoint's cost; the solver's roofline is "
                                 "reported on the large_pile line"},
            "cpu_baseline": cpu,
            "e2e": {"value": world_size * units / (e2e / 1000.0), "unit": METRIC,
                    "h2d_bytes_per_step": 12 * (n + 1) / args.rollout_steps,
                    "d2h_bytes_per_step": (52 + 64) * (n + 1) / args.rollout_steps,
                    "timing": "host wall clock around the recorded rollout, the final-state readback and the "
                              "VJP (cotangents host->device, gradients device->host)"},
            "clocks": clocks, "gpu_launches": int(np.mean(launches)) if launches else 0,
        }
        print(json.dumps(line), flush=True)


def run_one_world_at_a_time(args, local_rank, kw, sample=64, steps=100):
    """The batch's alternative on the same GPU: each world as a world of its own, stepped one
    at a time through the plain path. Times ``steps`` steps (after the warm-up) of ``sample``
    worlds spread over the batch with CUDA events and reports their aggregate throughput."""
    import torch
    from natsel_b200 import scenes
    from natsel_b200.world import World, default_world_def
    s = scenes.WORLD_SETTINGS["batched_worlds"]
    units, ms = 0, 0.0
    picks = [int(k * kw["count"] / sample) for k in range(sample)]
    for k in picks:
        w = World(default_world_def(gravity=s["gravity"], enable_continuous=int(s["enable_continuous"]), device=local_rank))
        info = scenes.batch_world(w, k, kw["seed"])
        for _ in range(args.warmup):
            w.step(DT, 4)
        w.synchronize()
        stream = torch.cuda.ExternalStream(w.stream(), device=torch.device("cuda", local_rank))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            w.step(DT, 4)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        units += info["dynamic_bodies"] * 4 * steps
        w.close()
    return {"value": units / (ms / 1000.0), "unit": METRIC, "sample_worlds": sample, "steps_each": steps,
            "timing": "CUDA events around each world's steps, worlds run one after another"}


def run_e2e(args, local_rank, dev, barrier, reduce, world_size):
    """The same workload through the public API with host buffers: every step uploads that
    step's external forces and torques (24 B per body, host->device) and reads the whole body
    state back into pinned host memory (64 B per body)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    world, info, sub = build_gpu_world(args, local_rank)
    n = world.body_count
    rng = np.random.Generator(np.random.PCG64(17))
    forces = [rng.normal(0.0, 1.0, (n, 3)).astype(np.float32) for _ in range(8)]
    torques = [rng.normal(0.0, 0.1, (n, 3)).astype(np.float32) for _ in range(8)]
    pos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    rot = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    lin = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    ang = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)

    def one(k):
        world.apply_forces(forces[k % 8], torques[k % 8])
        world.step(DT, sub)
        world.get_bodies_into(pos, rot, lin, ang)

    for k in range(args.warmup):
        one(k)
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        one(k)
    barrier()
    value, ms = job_throughput(info["dynamic_bodies"], sub, args.steps, 1000.0 * (time.perf_counter() - t0), reduce)
    seconds = ms / 1000.0
    world.close()
    return {"value": value, "unit": METRIC,
            "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 64 * n, "ms_per_step": 1000.0 * seconds / args.steps,
            "timing": "host wall clock around the K steps, synchronised by each step's readback"}


def main(argv=None):
    args = parse_args(argv)
    if args.warmup < 1 or args.steps < 1:
        raise SystemExit("bench.py: need --steps >= 1 and --warmup >= 1")
    if args.impl == "reference":
        if int(os.environ.get("RANK", "0")) != 0:
            return  # the CPU reference runs once, on rank 0
        run_reference_arm(args)
    else:
        run_natsel_arm(args)


if __name__ == "__main__":
    main()
