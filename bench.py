#!/usr/bin/env python
"""Throughput of the rigid-body step (body-substeps per second) on one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl natsel|reference]

Workload (default): the 10 000-body pile, i.e. 6 000 boxes, 2 500 spheres and 1 500 capsules
dropped from a 40 x 60 x 40 m volume onto a ground box, stepped at 60 Hz with 4 substeps in
FP32 for 600 steps (scene builder ``natsel_b200.scenes.large_pile``; seeded synthetic data). A
step is one ``World::step`` (solver_integration.rs:807 in the reference): broadphase pair
update, narrowphase, colouring, prepare, the substep solve and finalize.

Timed steps: the K timed steps are spread evenly over the workload's whole run (600 steps of
the pile): after W untimed warm-up steps, every stride-th step is timed, stride =
max(1, (length - W) // K), and the steps between are run untimed. Both arms time the same
step numbers, listed in ``config.timed_steps``. With K >= length - W every step after the
warm-up is timed.

natsel arm (default): one world per GPU (replicas, weak scaling; no collective on the data
path). ``value`` is the device time of the K timed steps measured with CUDA events on the
world's stream, with the L2 flushed before each timed step outside the events (the working
set fits in L2); ``e2e`` repeats the schedule through the public C ABI with per-step host
inputs (external forces, copied host->device) and the full body state read back to pinned
host memory at every timed step. ``roofline`` is for the persistent solver kernel (k_solve):
algorithmic bytes per launch from the per-step solver counts divided by its CUDA-event
duration. ``cpu_baseline`` times the CPU oracle (a scalar C++ restatement of the reference
step, -O3 -march=native built on this host) on one thread over a subset of the same timed
steps. The other parts of the metric ride on the same line as sub-records, each on its own
workload: ``batched_worlds`` (4 096 uneven worlds stepped together, against the same worlds
stepped one at a time on the same GPU, with the launch-shape autotuner's table; over N ranks
the worlds are split by body count, no exchange), ``jointed_chains`` (2 000 capsule chains on
revolute joints plus 4 000 boxes, 8 substeps, sampled over its 500 steps, with its solver
roofline) and ``differentiable_rollout`` (forward and adjoint ms/step of the 1 024-cube
rollout, with finite-difference and f64 checks).

reference arm (``--impl reference``): the reference engine is Rust and cannot be built on
this image, so its CPU step is timed through the oracle port, built -O3 -march=native on this
host: one world colour-parallel on every host core, as the reference parallelises a world,
over the same timed steps (``--reference-mode replicas``: one replica world per core
instead; batched worlds always run one world per core); under torchrun only rank 0 runs it.
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
# steps of each workload's run; the timed steps are spread over it
LENGTHS = {"large_pile": 600, "box_pyramid": 1000, "large_pyramid": 200, "batched_worlds": 1000,
           "jointed_chains": 500, "differentiable_rollout": 64}
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
    ap.add_argument("--no-subrecords", action="store_true",
                    help="skip the batched-worlds, jointed-chains and differentiable-rollout sub-records")
    ap.add_argument("--shapes", default=None,
                    help="launch shapes as JSON (the keys of World.launch_shapes()) instead of the autotuner's "
                         "choice, for profiling a fixed configuration")
    ap.add_argument("--sub-steps", type=int, default=10,
                    help="timed steps of each sampled sub-record (batched worlds, jointed chains)")
    return ap.parse_args(argv)


def timed_schedule(length, steps, warmup):
    """1-based numbers of the K timed steps: every stride-th step from W + 1, with stride =
    max(1, (length - W) // K), so the K steps cover the workload's whole run (K is capped at the
    length - W steps the run has after the warm-up)."""
    steps = max(1, min(steps, length - warmup))
    stride = max(1, (length - warmup) // steps)
    return [warmup + 1 + k * stride for k in range(steps)]


def schedule_block(schedule, length):
    stride = schedule[1] - schedule[0] if len(schedule) > 1 else 1
    return {"count": len(schedule), "first": schedule[0], "last": schedule[-1], "stride": stride,
            "run_length": length, "steps": schedule if len(schedule) <= 64 else None}


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


def profiled_traffic(algorithmic_bytes, kernel_file="k_solve_large_pile.json"):
    """DRAM bytes per solver launch from the committed ncu capture of k_solve on this workload
    (profiles/k_solve_large_pile.json: dram__bytes_read.sum + dram__bytes_write.sum and the
    launch's algorithmic bytes), scaled to this run by algorithmic bytes; None without it."""
    path = os.path.join(ROOT, "profiles", kernel_file)
    try:
        with open(path) as f:
            rec = json.load(f)
        t, a = float(rec["traffic_bytes_per_launch"]), float(rec["algorithmic_bytes_per_launch"])
    except (OSError, ValueError, KeyError):
        return None, None
    if a <= 0:
        return None, None
    return t / a * algorithmic_bytes, rec.get("capture", kernel_file)


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
# CPU side (oracle): single-thread baseline and the reference arm

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


_ORACLE_BUILD = None


def oracle_timing_build():
    """Load the oracle's timing build (-O3 -march=native for this host) once per process."""
    global _ORACLE_BUILD
    if _ORACLE_BUILD is None:
        from oracle import pyoracle
        _ORACLE_BUILD = pyoracle.use_host_native()
    return _ORACLE_BUILD


def thin(schedule, most):
    """At most ``most`` entries of the schedule, evenly spaced, first and last kept."""
    if len(schedule) <= most:
        return list(schedule)
    idx = sorted({round(k * (len(schedule) - 1) / (most - 1)) for k in range(most)})
    return [schedule[i] for i in idx]


def oracle_sampled(scene, kw, schedule, timed_threads, untimed_threads, budget_s):
    """Step one oracle world through the schedule: the steps between timed ones on
    ``untimed_threads`` host threads, each timed step on ``timed_threads``; stops after the
    budget (the timed steps done so far are reported)."""
    from natsel_b200 import scenes
    from oracle import pyoracle
    oracle_timing_build()
    sub = scenes.SUBSTEPS[scene]
    w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[scene])
    info = scenes.BUILDERS[scene](w, **kw)
    done, seconds, timed = 0, 0.0, []
    t_start = time.perf_counter()
    for target in schedule:
        pyoracle.set_threads(untimed_threads)
        while done < target - 1:
            w.step(DT, sub)
            done += 1
        pyoracle.set_threads(timed_threads)
        t0 = time.perf_counter()
        w.step(DT, sub)
        seconds += time.perf_counter() - t0
        done += 1
        timed.append(target)
        if time.perf_counter() - t_start > budget_s:
            break
    pyoracle.set_threads(1)
    return {"steps": len(timed), "timed": timed, "seconds": seconds, "bodies": info["dynamic_bodies"],
            "substeps": sub, "value": len(timed) * info["dynamic_bodies"] * sub / seconds}


def oracle_batch_run(kw, warmup, max_steps, budget_s, barrier=None, first_world=0, world_step=1):
    """The oracle on the batch, world by world (the oracle is one world): worlds first_world,
    first_world + world_step, ... each run warmup + max_steps steps, until the budget is spent."""
    from natsel_b200 import scenes
    from oracle import pyoracle
    oracle_timing_build()
    if barrier is not None:
        barrier.wait()
    units, seconds, steps, k = 0, 0.0, 0, first_world
    while seconds < budget_s and k < kw["count"]:
        w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS["batched_worlds"])
        info = scenes.batch_world(w, k, kw["seed"])
        for _ in range(warmup):
            w.step(DT, 4)
        t0 = time.perf_counter()
        for _ in range(max_steps):
            w.step(DT, 4)
        seconds += time.perf_counter() - t0
        units += info["dynamic_bodies"] * 4 * max_steps
        steps += max_steps
        k += world_step
    return {"steps": steps, "seconds": seconds, "units": units, "worlds": (k - first_world) // world_step}


def oracle_replica(scene, kw, schedule, budget_s, barrier=None):
    """One replica world on one thread over the schedule (the replicas mode of the reference arm)."""
    from natsel_b200 import scenes
    from oracle import pyoracle
    oracle_timing_build()
    sub = scenes.SUBSTEPS[scene]
    w = pyoracle.OracleWorld(**scenes.WORLD_SETTINGS[scene])
    info = scenes.BUILDERS[scene](w, **kw)
    for _ in range(schedule[0] - 1):
        w.step(DT, sub)
    if barrier is not None:
        barrier.wait()
    r = oracle_sampled_from(w, sub, schedule, budget_s)
    r.update(bodies=info["dynamic_bodies"], substeps=sub)
    return r


def oracle_sampled_from(w, sub, schedule, budget_s):
    done, seconds, timed = schedule[0] - 1, 0.0, []
    t_start = time.perf_counter()
    for target in schedule:
        while done < target - 1:
            w.step(DT, sub)
            done += 1
        t0 = time.perf_counter()
        w.step(DT, sub)
        seconds += time.perf_counter() - t0
        done += 1
        timed.append(target)
        if time.perf_counter() - t_start > budget_s:
            break
    return {"steps": len(timed), "timed": timed, "seconds": seconds}


def _replica_worker(kind, args_, barrier, queue):
    try:
        if kind == "batch":
            kw, warmup, steps, budget, first, stride = args_
            queue.put(oracle_batch_run(kw, warmup, steps, budget, barrier, first, stride))
        else:
            queue.put(oracle_replica(args_[0], args_[1], args_[2], args_[3], barrier))
    except Exception as e:  # report instead of hanging the parent
        queue.put({"error": repr(e)})


def run_reference_arm(args):
    from oracle import pyoracle
    pyoracle.build()
    scene, kw, desc = WORKLOADS[args.workload]
    n = min(host_cores(), 128)
    schedule = timed_schedule(LENGTHS[scene], args.steps, args.warmup)
    if scene != "batched_worlds" and args.reference_mode == "colour-parallel":
        return run_reference_colour_parallel(args, scene, kw, desc, n, schedule)
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(n)
    queue = ctx.Queue()
    if scene == "batched_worlds":
        jobs = [("batch", (kw, args.warmup, args.steps, args.reference_seconds, r, n)) for r in range(n)]
    else:
        jobs = [("replica", (scene, kw, schedule, args.reference_seconds)) for _ in range(n)]
    procs = [ctx.Process(target=_replica_worker, args=(kind, a, barrier, queue)) for kind, a in jobs]
    for p in procs:
        p.start()
    results = [queue.get(timeout=args.reference_seconds + 900) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    errors = [r["error"] for r in results if "error" in r]
    if errors:
        raise RuntimeError("reference replica failed: %s" % errors[0])
    seconds = max(r["seconds"] for r in results)
    if scene == "batched_worlds":
        units = sum(r["units"] for r in results)
        ms_per_step = 1000.0 * statistics.mean(r["seconds"] / max(r["steps"], 1) for r in results)
        sample = ("%d processes (one per host core, %s) stepping the batch's worlds one after another, "
                  "%d worlds, steps %d..%d of each (bounded to %.0f s); oracle build: %s" % (
                      n, cpu_model(), sum(r.get("worlds", 0) for r in results), args.warmup + 1,
                      args.warmup + args.steps, args.reference_seconds, oracle_build_note()))
        timed = None
    else:
        units = sum(r["steps"] * r["bodies"] * r["substeps"] for r in results)
        ms_per_step = 1000.0 * statistics.mean(r["seconds"] / r["steps"] for r in results)
        timed = min((r["timed"] for r in results), key=len)
        sample = ("%d replica worlds (one per host core, %s), each timing steps %s of the run (bounded to "
                  "%.0f s); oracle build: %s" % (n, cpu_model(), _steps_text(timed), args.reference_seconds,
                                                 oracle_build_note()))
    value = units / seconds
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene builder, no dataset)",
        "config": config_block(args, desc, schedule, scene), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_steps_done": timed,
    }
    print(json.dumps(line), flush=True)


def oracle_build_note():
    return _ORACLE_BUILD or "portable -O3 build"


def _steps_text(timed):
    if not timed:
        return "none"
    if len(timed) == 1:
        return str(timed[0])
    return "%d..%d every %d (%d steps)" % (timed[0], timed[-1], timed[1] - timed[0], len(timed))


def run_reference_colour_parallel(args, scene, kw, desc, n, schedule):
    """One world, as the reference steps it: the oracle's colour-parallel loops (collide per
    contact, prepare and every solver stage per constraint of a colour, the body stages per body;
    the pair update, the ordered state pass and the overflow colour stay serial) on every host
    core, timing the schedule's steps within the time budget."""
    r = oracle_sampled(scene, kw, schedule, n, n, args.reference_seconds)
    sample = ("one world, colour-parallel on %d host threads (%s), timed steps %s of the %d-step run (bounded "
              "to %.0f s); oracle build: %s" % (n, cpu_model(), _steps_text(r["timed"]), LENGTHS[scene],
                                                args.reference_seconds, oracle_build_note()))
    line = {
        "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * r["seconds"] / r["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene builder, no dataset)",
        "config": config_block(args, desc, schedule, scene), "impl": "reference",
        "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": n, "kind": "port", "sample": sample},
        "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_steps_done": r["timed"],
    }
    print(json.dumps(line), flush=True)


def config_block(args, desc, schedule, scene):
    par = "replicas: one independent world per GPU (%d)" % args.gpus
    if scene == "batched_worlds":
        par = "the batch's worlds split over %d GPU(s) by body count (no exchange)" % args.gpus
    return {"workload": "%s: %s" % (args.workload, desc), "timed_steps": schedule_block(schedule, LENGTHS[scene]),
            "l2": "flushed before each timed step (256 MiB write outside the timed events)", "parallelism": par}


# ---------------------------------------------------------------------------------------------
# natsel arm

def build_gpu_world(scene, kw, device, indices=None):
    from natsel_b200 import scenes
    from natsel_b200.world import World, default_world_def
    s = scenes.WORLD_SETTINGS[scene]
    w = World(default_world_def(gravity=s["gravity"], enable_continuous=int(s["enable_continuous"]), device=device))
    if indices is not None:
        info = scenes.batched_worlds(w, indices=indices, **kw)
    else:
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


def batch_share(kw, rank, world_size):
    """This rank's worlds of the batch: the body-count-balanced partition (natsel_b200.partition)."""
    from natsel_b200 import scenes
    from natsel_b200.partition import partition_worlds
    sizes = [scenes.batch_world_size(k, kw["seed"]) for k in range(kw["count"])]
    return partition_worlds(sizes, world_size)[rank]


class Ctx:
    """Per-rank plumbing of the natsel arm."""

    def __init__(self, rank, local_rank, world_size, dev, uuids):
        import torch
        self.rank, self.local_rank, self.world_size, self.dev, self.uuids = rank, local_rank, world_size, dev, uuids
        self.reduce = make_reducer(world_size, dev)
        self.flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def barrier(self):
        import torch
        import torch.distributed as dist
        if self.world_size > 1:
            dist.barrier()
        torch.cuda.synchronize()


def measure_device(ctx, world, sub, schedule, sample_clocks):
    """Run the schedule on ``world`` (already built, not yet stepped): untimed steps up to each
    timed one, the L2 flushed, then the timed step between CUDA events on the world's stream.
    Returns per-timed-step arrays and the clocks seen during the timed region."""
    import numpy as np
    import torch
    for _ in range(schedule[0] - 1):
        world.step(DT, sub)
    world.synchronize()
    stream = torch.cuda.ExternalStream(world.stream(), device=ctx.dev)  # created by the first step
    k_steps = len(schedule)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(k_steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(k_steps)]
    phase = np.zeros((k_steps, 5), np.float64)
    solve_bytes = np.zeros(k_steps, np.float64)
    launches = np.zeros(k_steps, np.int64)
    counts = np.zeros((k_steps, 4), np.float64)
    phases = np.zeros(k_steps, np.float64)
    ctx.barrier()
    sampler = ClockSampler(ctx.uuids) if (ctx.rank == 0 and sample_clocks) else None
    wall0 = time.perf_counter()
    done = schedule[0] - 1
    with torch.cuda.stream(stream):
        for k, target in enumerate(schedule):
            while done < target - 1:
                world.step(DT, sub)
                done += 1
            ctx.flush.zero_()
            # an NVTX range marks each timed step, so a profiler can list exactly these launches
            # (ncu --nvtx --nvtx-include "timed_step/")
            torch.cuda.nvtx.range_push("timed_step")
            starts[k].record(stream)
            world.step(DT, sub)
            ends[k].record(stream)
            torch.cuda.nvtx.range_pop()
            ends[k].synchronize()
            done += 1
            phase[k] = world.phase_times()
            sc = world.solver_counts()
            solve_bytes[k] = solve_launch_bytes(sc, sub)
            launches[k] = int(sc[11])
            phases[k] = float(sc[15])
            c = world.counters()
            counts[k] = (c[0], c[1], sc[2], sc[5])
    world.synchronize()
    ctx.barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop() if sampler else None
    step_ms = np.array([s_.elapsed_time(e) for s_, e in zip(starts, ends)])
    return {"step_ms": step_ms, "phase": phase, "solve_bytes": solve_bytes, "launches": launches,
            "counts": counts, "clocks": clocks, "wall": wall, "solve_phases": phases}


def latency_floor(ctx, world_kw, substeps=4, solver_blocks=None, steps=60):
    """The solver's per-phase floor: the time of one dependent phase (the barrier over the launch
    plus one constraint's load-and-solve chain) measured on a world with one box resting on a
    ground box, whose launch is 4 phases per substep with one item each. Returns us per phase."""
    from natsel_b200.world import World, default_world_def
    kw = dict(world_kw)
    if solver_blocks is not None:
        kw["solver_blocks"] = solver_blocks
    w = World(default_world_def(device=ctx.local_rank, **kw))
    g = w.create_body(type=0, position=(0.0, -0.5, 0.0))
    w.create_box(g, 5.0, 0.5, 5.0)
    b = w.create_body(type=2, position=(0.0, 0.5, 0.0))
    w.create_box(b, 0.5, 0.5, 0.5)
    for _ in range(10):
        w.step(DT, substeps)
    ms, ph = 0.0, 0
    for _ in range(steps):
        w.step(DT, substeps)
        ms += float(w.phase_times()[3])
        ph += int(w.solver_counts()[15])
    w.close()
    return 1000.0 * ms / max(ph, 1)


def roofline_block(m, kernel="k_solve", traffic_file="k_solve_large_pile.json", floor_us=None):
    solve_ms = m["phase"][:, 3]
    achieved = m["solve_bytes"].sum() / (solve_ms.sum() / 1000.0) / 1e9
    peak, peak_kind = measured_peak()
    alg = float(m["solve_bytes"].mean())
    traffic, source = profiled_traffic(alg, traffic_file) if traffic_file else (None, None)
    rec = {"kernel": kernel, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
           "frac": achieved / peak, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
           if peak_kind == "measured" else peak_kind,
           "traffic": traffic, "traffic_source": source,
           "algorithmic_bytes_per_launch": alg, "launch_ms": float(solve_ms.mean())}
    if floor_us is not None:
        # the latency roofline the launch actually meets: its dependent phases times the measured
        # floor of one phase (barrier plus one constraint's chain, one item per phase)
        ph = float(m["solve_phases"].mean())
        floor_ms = ph * floor_us / 1000.0
        rec["latency"] = {"phases_per_launch": ph, "floor_us_per_phase": floor_us, "floor_ms": floor_ms,
                          "frac": floor_ms / float(solve_ms.mean()),
                          "us_per_phase": 1000.0 * float(solve_ms.mean()) / ph if ph else None,
                          "floor_method": "one box resting on a ground box, same solver launch shape: "
                                          "solve time / its phases (4 per substep, one item each)"}
    return rec


def step_counts_block(m):
    c = m["counts"].mean(0)
    return {"live_contacts": float(c[0]), "touching_contacts": float(c[1]), "coloured_manifolds": float(c[2]),
            "joints": float(c[3])}


def measure_e2e(ctx, scene, kw, schedule, indices=None, warmup=0, shapes=None):
    """The schedule through the public API with host buffers: every step uploads that step's
    external forces and torques (24 B per body, host->device); every timed step also reads the
    whole body state back into pinned host memory (64 B per body). The wall clock of each timed
    step (forces, step, readback) is summed; the steps between run untimed."""
    import numpy as np
    import torch
    world, info, sub = build_gpu_world(scene, kw, ctx.local_rank, indices)
    n = world.body_count
    rng = np.random.Generator(np.random.PCG64(17))
    forces = [rng.normal(0.0, 1.0, (n, 3)).astype(np.float32) for _ in range(8)]
    torques = [rng.normal(0.0, 0.1, (n, 3)).astype(np.float32) for _ in range(8)]
    pos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    rot = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
    lin = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    ang = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    if shapes is not None:
        world.set_launch_shapes(shapes)  # the same launch shapes as the device-timed run
    done, seconds = 0, 0.0
    while done < warmup:
        world.apply_forces(forces[done % 8], torques[done % 8])
        world.step(DT, sub)
        done += 1
    ctx.barrier()
    for target in schedule:
        while done < target - 1:
            world.apply_forces(forces[done % 8], torques[done % 8])
            world.step(DT, sub)
            done += 1
        world.synchronize()
        t0 = time.perf_counter()
        world.apply_forces(forces[done % 8], torques[done % 8])
        world.step(DT, sub)
        world.get_bodies_into(pos, rot, lin, ang)
        seconds += time.perf_counter() - t0
        done += 1
    ctx.barrier()
    value, ms = job_throughput(info["dynamic_bodies"], sub, len(schedule), 1000.0 * seconds, ctx.reduce)
    world.close()
    return {"value": value, "unit": METRIC, "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 64 * n,
            "ms_per_step": ms / len(schedule),
            "timing": "host wall clock of each timed step (force upload, step, full body-state readback), "
                      "summed over the same timed steps"}


def run_natsel_arm(args):
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
    uuids = [str(torch.cuda.get_device_properties(local_rank).uuid)]
    if world_size > 1:
        gathered = [None] * world_size
        dist.all_gather_object(gathered, uuids[0])
        uuids = gathered
    ctx = Ctx(rank, local_rank, world_size, dev, uuids)
    try:
        scene, kw, desc = WORKLOADS[args.workload]
        if scene == "differentiable_rollout":
            line = measure_rollout(args, ctx, args.steps, args.warmup, with_checks=not args.no_cpu_baseline)
            if rank == 0:
                line.update({"config": {
                    "workload": "%s: %s" % (args.workload, desc),
                    "timed_steps": "%d rollouts of %d steps" % (args.steps, args.rollout_steps),
                    "l2": "working set (~40 MB of world and tape) stays in L2 between rollouts; not flushed",
                    "parallelism": "replicas: one independent world per GPU (%d)" % args.gpus}})
                print(json.dumps(line), flush=True)
            return
        if scene == "batched_worlds":
            line = measure_batched(args, ctx, kw, args.steps, args.warmup, headline=True)
        else:
            line = measure_plain(args, ctx, scene, kw, desc, args.steps, args.warmup, headline=True)
        if scene == "large_pile" and not args.no_subrecords:
            sub_k = max(1, args.sub_steps)
            b_kw = WORKLOADS["batched_worlds"][1]
            line["batched_worlds"] = measure_batched(args, ctx, b_kw, sub_k, 3, headline=False)
            c_scene, c_kw, c_desc = WORKLOADS["jointed_chains"]
            chains = measure_plain(args, ctx, c_scene, c_kw, c_desc, sub_k, args.warmup, headline=False)
            line["jointed_chains"] = chains
            rollout = measure_rollout(args, ctx, 2, 1, with_checks=not args.no_cpu_baseline)
            line["differentiable_rollout"] = rollout
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world_size > 1:
            dist.barrier()
            dist.destroy_process_group()


def measure_plain(args, ctx, scene, kw, desc, steps, warmup, headline):
    """One world per rank over the sampled schedule: device timing, roofline, e2e and (headline,
    one rank) the one-thread CPU baseline. Returns the JSON record (rank 0) or None."""
    length = LENGTHS[scene]
    schedule = timed_schedule(length, steps, warmup)
    indices = batch_share(kw, ctx.rank, ctx.world_size) if scene == "batched_worlds" else None
    # launch shapes for this workload (solver, recycle pass, manifold updates, preparation), each
    # timed from a copy of a world's state by the autotuner. A single world is tuned on a copy of
    # the scene stepped to the middle of its run (the drop's first steps hold few contacts), and
    # the measured world takes those shapes; a batch is tuned on itself after the warm-up.
    world, info, sub = build_gpu_world(scene, kw, ctx.local_rank, indices)
    if scene == "batched_worlds":
        tune_step = warmup
        for _ in range(warmup):
            world.step(DT, sub)
        autotune = [{"blocks": b, "cooperative_grid": g, "ms_per_step": ms}
                    for b, g, ms in world.autotune(DT, sub, 3)]
        tune_rows, shapes = world.autotune_table(), world.launch_shapes()
        done = warmup
    elif args.shapes and headline:
        tune_step, autotune, tune_rows = None, None, None
        shapes = dict(world.launch_shapes(), **json.loads(args.shapes))
        world.set_launch_shapes(shapes)
        for _ in range(warmup):
            world.step(DT, sub)
        done = warmup
    else:
        tune_step = length // 2
        tw, _, _ = build_gpu_world(scene, kw, ctx.local_rank, indices)
        for _ in range(tune_step):
            tw.step(DT, sub)
        autotune = [{"blocks": b, "cooperative_grid": g, "ms_per_step": ms} for b, g, ms in tw.autotune(DT, sub, 3)]
        tune_rows, shapes = tw.autotune_table(), tw.launch_shapes()
        tw.close()
        world.set_launch_shapes(shapes)
        for _ in range(warmup):
            world.step(DT, sub)
        done = warmup
    schedule = [s_ for s_ in schedule if s_ > warmup] or [warmup + 1]
    m = measure_device_continue(ctx, world, sub, schedule, done, sample_clocks=headline)
    world.close()
    bodies = info["dynamic_bodies"]
    value, total_ms = job_throughput(bodies, sub, len(schedule), float(m["step_ms"].sum()), ctx.reduce)
    launches = int(ctx.reduce(float(m["launches"].sum()), "sum"))
    traffic_file = "k_solve_large_pile.json" if scene == "large_pile" else None
    from natsel_b200 import scenes as _scenes
    s_ = _scenes.WORLD_SETTINGS[scene]
    floor_us = latency_floor(ctx, {"gravity": s_["gravity"], "enable_continuous": int(s_["enable_continuous"])},
                             sub, solver_blocks=shapes["solver_blocks"] if shapes["solver_grid"] else
                             min(shapes["solver_blocks"], 16))
    rec = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ctx.world_size, "steps": len(schedule),
        "warmup": warmup, "ms_per_step": total_ms / len(schedule), "higher_is_better": True,
        "scaling": "strong" if scene == "batched_worlds" else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene builder, no dataset)",
        "config": config_block(args, desc, schedule, scene) if headline else
        {"workload": "%s: %s" % (scene, desc), "timed_steps": schedule_block(schedule, length),
         "l2": "flushed before each timed step (256 MiB write outside the timed events)"},
        "roofline": roofline_block(m, traffic_file=traffic_file, floor_us=floor_us),
        "clocks": m["clocks"], "gpu_launches": launches, "wall_s": m["wall"],
        "phase_ms_mean": {k: float(v) for k, v in zip(["broadphase", "collide", "state_color_prepare", "solve",
                                                      "finalize"], m["phase"].mean(0))},
        "step_counts_mean": step_counts_block(m), "dynamic_bodies": bodies,
    }
    rec["solver_autotune"] = autotune
    rec["autotune"] = {"chosen": shapes, "candidates": tune_rows, "tuned_at_step": tune_step,
                       "method": "each candidate steps 1 + 3 steps from a copy of the world's state at the "
                                 "tuning step, CUDA events; one kernel at a time, the fastest kept; the world "
                                 "is restored, and the measured world takes the chosen shapes"
                                 if autotune is not None else "fixed by --shapes"}
    if headline and not args.no_e2e:
        rec["e2e"] = measure_e2e(ctx, scene, kw, schedule, indices, warmup, shapes)
    if headline and ctx.rank == 0 and ctx.world_size == 1 and not args.no_cpu_baseline and scene == "batched_worlds":
        r = oracle_batch_run(kw, warmup, steps, args.cpu_seconds)
        rec["cpu_baseline"] = {
            "value": r["units"] / r["seconds"], "unit": METRIC, "cores": 1, "kind": "port",
            "sample": "CPU oracle (%s) on 1 thread (%s): %d of the batch's worlds one after another, steps "
                      "%d..%d of each (bounded to %.0f s)" % (oracle_build_note(), cpu_model(), r["worlds"],
                                                              warmup + 1, warmup + steps, args.cpu_seconds)}
    elif headline and ctx.rank == 0 and ctx.world_size == 1 and not args.no_cpu_baseline:
        cpu_sched = thin(schedule, 40)
        r = oracle_sampled(scene, kw, cpu_sched, 1, host_cores(), args.cpu_seconds)
        rec["cpu_baseline"] = {
            "value": r["value"], "unit": METRIC, "cores": 1, "kind": "port",
            "sample": "CPU oracle (scalar C++ restatement of the reference step; %s) on 1 thread (%s), timing "
                      "steps %s of the same %d-step run, the steps between run untimed on every core "
                      "(bounded to %.0f s)" % (oracle_build_note(), cpu_model(), _steps_text(r["timed"]), length,
                                               args.cpu_seconds)}
    elif headline:
        rec["cpu_baseline"] = None
    return rec if ctx.rank == 0 else None


def measure_device_continue(ctx, world, sub, schedule, done, sample_clocks):
    """measure_device for a world that has already run ``done`` steps."""
    shifted = [s_ - done for s_ in schedule]
    return measure_device(ctx, world, sub, shifted, sample_clocks)


def measure_batched(args, ctx, kw, steps, warmup, headline):
    """The batched worlds: the batch (this rank's share) sampled over its 1000-step run, the
    autotuner's table, and the same worlds stepped one at a time on the same GPU."""
    scene, _, desc = WORKLOADS["batched_worlds"]
    rec = measure_plain(args, ctx, scene, kw, desc, steps, warmup, headline=headline)
    if ctx.rank == 0:
        one = run_one_world_at_a_time(args, ctx.local_rank, kw)
        rec["one_world_at_a_time"] = one
        rec["batched_over_one_at_a_time"] = rec["value"] / ctx.world_size / one["value"]
        rec["parallelism"] = "the 4 096 worlds split over %d GPU(s) by body count (no exchange)" % ctx.world_size
    return rec


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


def measure_rollout(args, ctx, reps, warmup, with_checks):
    """The differentiable rollout: per timed repetition, the plain forward rollout (64 steps, no
    tape), the same rollout recorded on a tape (checkpoint copies every 8 substeps) and its
    vector-Jacobian product, each timed with CUDA events on the world's stream. The value is
    body-substeps/s through the recorded forward plus the adjoint; the adjoint's cost is
    reported against the plain forward's. Returns the record (rank 0) or None."""
    import numpy as np
    import torch
    from natsel_b200 import scenes
    from natsel_b200.world import World, default_world_def
    s = scenes.WORLD_SETTINGS["differentiable_rollout"]
    rank, local_rank, dev = ctx.rank, ctx.local_rank, ctx.dev

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
    for rep in range(warmup + reps):
        timed = rep >= warmup
        if timed and sampler is None and rank == 0:
            ctx.barrier()
            sampler = ClockSampler(ctx.uuids)
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
        if timed and rep == warmup + reps - 1 and rank == 0 and with_checks:
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
    plain = ctx.reduce(float(np.mean(plain_ms)), "max")
    taped = ctx.reduce(float(np.mean(taped_ms)), "max")
    vjp = ctx.reduce(float(np.mean(vjp_ms)), "max")
    e2e = ctx.reduce(float(np.mean(e2e_ms)), "max")
    value = ctx.world_size * units / ((taped + vjp) / 1000.0)
    fd = rollout_fd_check(args, local_rank, grads) if (rank == 0 and with_checks) else None
    cpu = None
    if rank == 0 and ctx.world_size == 1 and with_checks:
        sched = list(range(2, args.rollout_steps + 2))
        r = oracle_sampled("differentiable_rollout", {}, sched, 1, 1, args.cpu_seconds)
        cpu = {"value": r["value"], "unit": METRIC, "cores": 1, "kind": "port",
               "sample": "CPU oracle forward rollout only (the reference has no adjoint), steps %s, 1 thread, %s; "
                         "oracle build: %s" % (_steps_text(r["timed"]), cpu_model(), oracle_build_note())}
    solve_ms = phase[3] / max(k, 1) / args.rollout_steps
    if rank != 0:
        return None
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": ctx.world_size, "steps": reps,
        "warmup": warmup, "ms_per_step": (taped + vjp) / args.rollout_steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene builder, no dataset)",
        "config": {"workload": "differentiable_rollout: %s" % WORKLOADS["differentiable_rollout"][2],
                   "timed_steps": "%d rollouts of %d steps" % (reps, args.rollout_steps)},
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
        "e2e": {"value": ctx.world_size * units / (e2e / 1000.0), "unit": METRIC,
                "h2d_bytes_per_step": 12 * (n + 1) / args.rollout_steps,
                "d2h_bytes_per_step": (52 + 64) * (n + 1) / args.rollout_steps,
                "timing": "host wall clock around the recorded rollout, the final-state readback and the "
                          "VJP (cotangents host->device, gradients device->host)"},
        "clocks": clocks, "gpu_launches": int(np.mean(launches)) if launches else 0,
    }


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
        for _ in range(3):
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
            "timing": "CUDA events around steps 4..103 of each world, worlds run one after another"}


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
