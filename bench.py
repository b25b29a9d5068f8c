"""Benchmark: subsphere-steps/s of the NBodyClump step on a B200.

Workload (one GPU): the cfg1 bed -- 50,000 tetrahedral clumps = 200,000
subspheres (r = 1 mm x LogNormal(0, 0.2), centre offset 0.6 r, random
orientation) in a closed cylinder wall (R = 60 mm, half-height 150 mm),
contact law in FP32 with FP64 positions and quaternions, dt = 0.2 of the
Rayleigh step, Thresh = 0.2 r_min, 5 hierarchical-grid levels -- started from
its engine-settled state after 20,000 steps of settling under gravity
(tests/golden/cfg1_settled.npz, made by tests/golden/make_cfg1_state.py), so
every timed step has touching pairs, wall contacts and list rebuilds.  One
step = one pass of the clump step (kick/drift/attitude/pose, list rebuild
when triggered, contacts, clump reduction).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

The default line also carries a `batched` record: the first 64 scenes of
the cfg3 draw (cfg1-style beds, clump counts log-uniform in [500, 50,000],
friction U[0.2, 0.8]), settled together for 2,000 steps, then advanced 300
steps as one batch against the same scenes one at a time on the plain
engine (the batched-vs-plain metric on a fixed subset).

Under torchrun each rank runs its own replica of the workload: weak
scaling, no collective on the data path; timing is the max over ranks.
Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
# concurrent scene streams (batch and serving modes) need more than the default
# 8 hardware work queues; read by CUDA when the process first uses it
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
sys.path.insert(0, os.path.join(REPO, "nbody-clump_b200"))
import scenegen as sg  # noqa: E402

METRIC = "subsphere-steps/sec"
SNAPSHOT = os.path.join(REPO, "tests", "golden", "cfg1_settled.npz")
WORKLOAD = ("cfg1: 50,000 tetra clumps (200,000 subspheres) in a closed cylinder wall (R 60 mm, half-height "
            "150 mm), from the engine-settled state after {steps} steps of settling")


def peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6553.6), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(value, world, backend):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if backend == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def replica_throughput(n_sub, steps, world, local_seconds, backend):
    """Whole-job throughput of `world` independent replicas (one scene per
    rank, the same work on each): the slowest rank's time, taken by an
    all-reduce, and units = n_sub x steps x world.  Returns (seconds, value)."""
    secs = reduce_max(local_seconds, world, backend)
    return secs, n_sub * steps * world / secs


def workload(args):
    """The benchmarked scene: the engine-settled cfg1 snapshot (its grid
    levels are stored with it, so neither arm needs the level chooser); with
    --scene, a scene saved by --save-state; with --from-seed, the cfg1 bed as
    seeded (falling, levels from nbc_choose_levels).  Returns (scene, config)
    where config describes the workload identically for both arms."""
    if args.scene:
        scene = sg.scene_from_npz(args.scene)
        start = f"scene file {os.path.basename(args.scene)}"
    elif args.from_seed:
        import nbc
        scene = nbc.with_levels(sg.make_cfg1(n_clumps=args.clumps, seed=20260828))
        start = "as seeded (loose layers, falling)"
    else:
        scene = sg.tetra_state_from_npz(SNAPSHOT)
        start = f"engine-settled state after {int(scene['meta']['steps'])} steps ({os.path.relpath(SNAPSHOT, REPO)})"
    N, K = int(scene["params"]["NumberBody"]), int(scene["params"]["ClumpNum"])
    lv = scene.get("levels")
    steps = int(scene.get("meta", {}).get("steps", 0))
    config = {"workload": WORKLOAD.format(steps=steps) if steps else WORKLOAD.split(", from")[0],
              "subspheres": N, "clumps": K, "grid_levels": 1 if lv is None else len(lv["cell"]),
              "start_state": start,
              "l2": "not flushed between steps: each step reads the state the previous step wrote "
                    "(~60 MB, resident in the 126 MB L2 as in real use)"}
    return scene, config


def run_b200(args, world, rank, local):
    import nbc
    backend = None
    if world > 1:
        import torch
        import torch.distributed as dist
        backend = "nccl"
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    scene, config = workload(args)
    N, K = config["subspheres"], config["clumps"]
    clk = ClockSampler(local)
    clk.__enter__()       # sampled over every GPU leg of the run (tuning, warm-up, timed region, replay, e2e)
    tuned = None
    if args.autotune:
        # launch shapes measured on this scene (results do not depend on them)
        tuned = nbc.autotune([scene], precision=args.precision, device=local, trial_steps=200)
    opts = dict(precision=args.precision, use_graph=args.graph, device=local, pair_slack=args.pair_slack,
                search_lanes=args.search_lanes, tuned=tuned)

    # ---- device-resident throughput -----------------------------------
    eng = nbc.Engine([scene], **opts)
    eng.step(args.warmup)
    eng.sync()
    st0 = eng.stats()
    # the timed region: no timing event nodes in the step graphs and no host
    # queries between its chunks (launches are still counted)
    launch = eng.launch_info()
    eng.timing_enable(2 if args.profile else 0)
    barrier(world)
    pair_samples = []
    t0 = time.perf_counter()
    left = args.steps
    while left > 0:           # each call returns after the device finished (stream synchronised)
        c = min(left, 1000)
        eng.step(c)
        if args.profile:
            pair_samples.append((c, eng.stats()["npairs"]) + eng.contact_counts())
        left -= c
    t1 = time.perf_counter()
    tm = eng.timing_read()
    st1 = eng.stats()
    barrier(world)
    local_s = t1 - t0
    secs, value = replica_throughput(N, args.steps, world, local_s, backend)
    launches = tm["kernel_launches"]
    if args.profile:
        clk.__exit__()
        if rank == 0:
            nt = eng.contact_counts()
            print(json.dumps({"profile_run": True, "ms_per_step": secs * 1e3 / args.steps,
                              "contact_ms_avg": tm["contact_ms"] / max(1, tm["contact_launches"]),
                              "npairs": st1["npairs"], "rebuilds": st1["rebuilds"] - st0["rebuilds"],
                              "phases_ms": eng.timing_phases(), "near_touching": nt,
                              "alg_bytes": algorithmic_contact_bytes(N, *nt, args.precision)}), flush=True)
        return
    # the kernels' CUDA-event times over a replay of the timed region (the
    # same scene, warm-up and steps on a second engine: runs are
    # deterministic, so it does the same work), with timing event nodes in
    # its step graphs, and the near and touching pair counts sampled every
    # chunk
    eng.close()
    eng = nbc.Engine([scene], **opts)
    eng.step(args.warmup)
    eng.sync()
    eng.timing_enable(2)
    left = args.steps
    chunk = max(1, min(1000, args.steps // 4))
    while left > 0:
        c = min(left, chunk)
        eng.step(c)
        pair_samples.append((c, eng.stats()["npairs"]) + eng.contact_counts())
        left -= c
    tm = eng.timing_read()
    phases = eng.timing_phases()
    eng.close()

    # ---- end to end through the C ABI with host buffers -----------------
    # create (H2D of the scene from host arrays), K steps, sync, D2H of the
    # clump state, all inside the timed region
    host_in = sum(np.asarray(v).nbytes for v in scene["sub"].values()) + \
        sum(np.asarray(v).nbytes for v in scene["clump"].values())
    barrier(world)
    te0 = time.perf_counter()
    e2 = nbc.Engine([scene], **opts)
    e2.step(args.warmup + args.steps)
    e2.sync()
    out = e2.clumps()
    te1 = time.perf_counter()
    e2.close()
    host_out = sum(v.nbytes for v in out.values())
    e2e_s = reduce_max(te1 - te0, world, backend)
    e2e_steps = args.warmup + args.steps
    e2e_value = N * e2e_steps * world / e2e_s

    # ---- the benchmarked law's per-contact forces at the start state (the
    # CPU-baseline leg compares them with the FP64 oracle) ----------------
    ex = nbc.Engine([scene], precision=args.precision, use_graph=False, device=local)
    ex.step_export(1)
    first_step = {"pairs": ex.pairs(), "fcn": ex.pair_forces()}
    ex.close()

    batched = None
    if rank == 0 and args.batch_scenes > 0:
        batched = batched_record(args)
    clk.__exit__()

    # ---- rooflines: the contact kernel and the clump pass --------------
    pk, pk_kind = peaks()
    wsum = max(1, sum(q[0] for q in pair_samples))
    npairs, nnear, ntouch = (sum(q[0] * q[i] for q in pair_samples) / wsum for i in (1, 2, 3))
    alg = algorithmic_contact_bytes(N, nnear, ntouch, args.precision)
    avg_ms = tm["contact_ms"] / max(1, tm["contact_launches"])
    achieved = alg / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else 0.0
    clump_ms = phases["clump"]
    alg_clump = algorithmic_clump_bytes(N, K, nnear, args.precision)
    clump_gbs = alg_clump / (clump_ms * 1e-3) / 1e9 if clump_ms > 0 else 0.0
    traffic, traffic_note = None, None
    tp = os.path.join(REPO, "profiles", "contact_traffic.json")
    if os.path.exists(tp):
        tj = json.load(open(tp))
        if tj.get("kernel") == "k_pairs" and tj.get("precision") == args.precision and tj.get("slots") == "entry":
            # captured on the same start state; scaled to this run's mean near
            # and touching pairs by the ratio of algorithmic bytes
            traffic = tj["dram_bytes_per_launch"] * alg / tj["algorithmic_bytes_at_capture"]
            traffic_note = tj["note"]

    cpu = cpu_baseline(args, scene, first_step) if (rank == 0 and not args.no_cpu_baseline) else None
    clocks = clk.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "subsphere-steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": secs * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 contact law, f64 positions/quaternions" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded numpy bed settled by the engine, no dataset)",
            "config": config,
            "engine": {"precision": args.precision, "graph": bool(args.graph), "autotuned": tuned, "launch": launch,
                       "pairs_listed_end": st1["npairs"],
                       "rebuilds_in_timed_region": st1["rebuilds"] - st0["rebuilds"],
                       "mean_pairs_near": nnear, "mean_pairs_touching": ntouch,
                       "parallelism": f"replicas x{world} (independent scenes)",
                       "phases_ms_per_step_replay": phases},
            "e2e": {"value": e2e_value, "unit": "subsphere-steps/s", "h2d_bytes_per_step": host_in / e2e_steps,
                    "d2h_bytes_per_step": host_out / e2e_steps, "steps": e2e_steps,
                    "includes": "nbc_create (upload) + first list build + steps + sync + clump-state download"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk, "unit": "GB/s",
                         "frac": achieved / pk if pk else None, "traffic": traffic,
                         "kernel": "contact pass (k_pairs)", "avg_launch_ms": avg_ms,
                         "alg_bytes_per_launch": alg, "mean_pairs_listed": npairs,
                         "mean_pairs_near": nnear, "mean_pairs_touching": ntouch, "peak_kind": pk_kind,
                         "window": "a replay of the timed region (same scene, warm-up and steps) with CUDA events "
                                   "on the engine's stream",
                         "traffic_note": traffic_note},
            "roofline_clump": {"bound": "hbm", "achieved": clump_gbs, "peak": pk, "unit": "GB/s",
                               "frac": clump_gbs / pk if pk else None, "kernel": "clump pass (k_clump)",
                               "avg_launch_ms": clump_ms, "alg_bytes_per_launch": alg_clump, "peak_kind": pk_kind},
            "cpu_baseline": cpu,
            "batched": batched,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def batched_record(args):
    """cfg3 on a fixed subset: the first --batch-scenes scenes of the cfg3
    draw, settled together for --batch-settle steps (untimed, so both arms
    start from the same contact-rich states), then --batch-steps steps as
    one batch (nbc_batch, launch shapes from the autotuner) against the same
    scenes one at a time on the plain engine (default shapes).  scenes/s
    includes engine creation (upload) and the first list build in both arms;
    subsphere-steps/s counts the stepping only."""
    import nbc
    scenes = [nbc.with_levels(x) for x in sg.make_cfg3(args.batch_scenes, steps=args.batch_steps)]
    n_sub = sum(int(x["params"]["NumberBody"]) for x in scenes)
    opts = dict(precision=args.precision, pair_slack=1.6)
    b = nbc.Batch(scenes, **opts)
    b.step(args.batch_settle)
    b.sync()
    states = [b.engines[i].restart_scene(scenes[i]) for i in range(len(scenes))]
    b.close()
    tuned = nbc.autotune(states, precision=args.precision, trial_steps=100) if args.autotune else None
    t0 = time.perf_counter()
    b = nbc.Batch(states, tuned=tuned, **opts)
    t1 = time.perf_counter()
    b.step(args.batch_steps)
    b.sync()
    t2 = time.perf_counter()
    reb_b = sum(v.stats()["rebuilds"] for v in b.engines)
    b.close()
    bc, bs = t1 - t0, t2 - t1
    pc = ps = 0.0
    for sc in states:
        t0 = time.perf_counter()
        e = nbc.Engine([sc], **opts)
        t1 = time.perf_counter()
        e.step(args.batch_steps)
        e.sync()
        ps += time.perf_counter() - t1
        pc += t1 - t0
        e.close()
    work = n_sub * args.batch_steps
    arm = lambda c, st: {"create_s": c, "step_s": st, "scenes_per_s": len(states) / (c + st),
                         "subsphere_steps_per_s": work / st}
    return {"metric": "subsphere-steps/s and scenes/s, batched vs plain (one at a time), same B200",
            "workload": f"first {len(states)} scenes of the cfg3 draw ({n_sub} subspheres), settled "
                        f"{args.batch_settle} steps together, then {args.batch_steps} steps timed",
            "batched": arm(bc, bs), "plain": arm(pc, ps), "rebuilds_batched": reb_b, "autotuned_batch": tuned,
            "speedup_steps": ps / bs, "speedup_scenes_per_s": (pc + ps) / (bc + bs)}


def save_state(args):
    """Advance the workload --advance steps and save the state it reached as a
    scene file (a starting point for short profiler runs)."""
    import nbc
    scene, _ = workload(args)
    eng = nbc.Engine([scene], precision=args.precision, use_graph=True)
    eng.step(args.advance)
    out = eng.restart_scene(scene)
    sg.scene_to_npz(out, args.save_state)
    print(json.dumps({"saved": args.save_state, "steps": args.advance, "npairs": eng.stats()["npairs"]}), flush=True)


def algorithmic_contact_bytes(N, nnear, ntouch, precision):
    """Unique bytes the contact kernel (k_pairs) must move per step.

    Per near pair (the pairs that can touch before the next rebuild, each
    visited once): its near front record (pair slot, partner, owner and near
    back slot, 16 B), both clump ids 8 B, the touch flag written 1 B, both subspheres' FP64
    position and radius 2 x 32 B, and the four contact slots written (force
    and torque on each side, 4 Real4).  Per touching pair: the previous touch
    flag 1 B, the spring history read and written (2 Real4 + 1 Real each way)
    and both subspheres' FP64 contact kinematics (3 x 32 B each: the
    subsphere's arm and mass, its clump's velocity and angular velocity).  N is unused: the
    per-subsphere sums are part of the clump pass."""
    r = 4 if precision == "mixed" else 8
    r4 = 4 * r
    per_near = 4 * 4 + 2 * 4 + 1 + 2 * 32 + 4 * r4
    per_touch = 1 + 2 * (2 * r4 + r) + 2 * 3 * 32
    return per_near * nnear + per_touch * ntouch


def algorithmic_clump_bytes(N, K, nnear, precision):
    """Unique bytes the clump pass (k_clump) must move per step: per clump
    its position, velocity, angular velocity, quaternion and properties read
    (5 x 32 B) and position, velocity, angular velocity, quaternion, force and
    torque written (6 x 32 B) plus its member offset 4 B; per member its index
    4 B, FP64 position read and written 2 x 32 B, body offset and mass 32 B,
    displacement since the rebuild read and written 2 x 32 B, contact
    kinematics (arm, mass) written 32 B, near-row offsets 16 B and boundary bits 2 B;
    per near pair its two contact-slot pairs read (4 Real4)."""
    r4 = 16 if precision == "mixed" else 32
    per_clump = 5 * 32 + 6 * 32 + 4
    per_sub = 4 + 2 * 32 + 32 + 2 * 32 + 32 + 16 + 2
    return per_clump * K + per_sub * N + 4 * r4 * nnear


def cpu_baseline(args, scene, first_step):
    """The FP64 CPU oracle on a bounded sample of the same workload, single
    thread.  Its first step (the list build) also checks the benchmarked
    engine's first step from the same state: the pair list bit for bit and
    every contact's normal force against FP64."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    threads = 1
    o = oracle.OracleScene(scene, threads=threads)
    o.step(1)  # first step includes the initial list build, like the GPU warm-up
    oa, ob = o.pairs()
    ea, eb = first_step["pairs"]
    same = bool(np.array_equal(oa, ea) and np.array_equal(ob, eb))
    err = None
    if same:
        fo = o.pair_caches()["cfcn"]
        fe = first_step["fcn"]
        mag = np.linalg.norm(fo, axis=1)
        big = mag > 1e-6 * mag.max() if mag.size else mag > 0
        rel = np.linalg.norm(fe - fo, axis=1)[big] / mag[big]
        err = {"max_rel_per_contact": float(rel.max()) if rel.size else 0.0, "contacts": int(big.sum()),
               "p99_rel": float(np.percentile(rel, 99)) if rel.size else 0.0, "tolerance": 1e-5,
               "law": args.precision}
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > args.cpu_seconds or n >= 200:
            break
    dt = time.perf_counter() - t0
    N = scene["params"]["NumberBody"]
    return {"value": N * n / dt, "unit": "subsphere-steps/s", "cores": threads, "kind": "port",
            "sample": f"{n} steps of the benchmarked {N}-subsphere scene from its start state, after its first "
                      "step (list build), single thread",
            "first_step_vs_engine": {"pair_list_bitexact": same, "force_error_vs_fp64": err}}


def run_batch(args):
    """cfg3: n independent cfg1-style scenes (clump counts log-uniform in
    [500, 50,000], friction U[0.2, 0.8], own seeds), advanced together
    (nbc_batch: one engine over all scenes, one launch per kernel and step,
    rebuilds over the scenes that need one) against the same scenes one at a
    time on the plain engine.  Both timings include engine creation (upload)
    and the first list build."""
    import nbc
    scenes = [nbc.with_levels(s) for s in sg.make_cfg3(args.scenes, steps=args.steps)]
    n_sub = sum(int(s["params"]["NumberBody"]) for s in scenes)
    opts = dict(precision=args.precision, pair_slack=1.6)
    if args.profile_window is not None:
        # for a launch list: eager launches (kernel nodes of a graph with a
        # conditional node are not profiled), the profiler range around
        # --steps steps after --profile-window steps
        import torch
        b = nbc.Batch(scenes, use_graph=False, **opts)
        b.step(args.profile_window)
        b.sync()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        b.step(args.steps)
        b.sync()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_run": True, "scenes": len(scenes), "subspheres": n_sub,
                          "window": [args.profile_window, args.profile_window + args.steps],
                          "rebuilds": sum(v.stats()["rebuilds"] for v in b.engines)}), flush=True)
        b.close()
        return
    # process start-up (CUDA context, lazy kernel loading) stays out of both arms
    w = nbc.Engine([scenes[0]], **opts)
    w.step(3)
    w.sync()
    w.close()
    # launch shapes for the batch measured on it (untimed); the plain arm keeps the defaults
    tuned = nbc.autotune(scenes, precision=args.precision, trial_steps=100) if args.autotune else None
    with ClockSampler(0) as clk_b:
        t0 = time.perf_counter()
        b = nbc.Batch(scenes, tuned=tuned, **opts)
        t1 = time.perf_counter()
        b.step(args.steps)
        b.sync()
        t2 = time.perf_counter()
    last = b.engines[0].clumps()
    b.close()
    bc, bs = t1 - t0, t2 - t1
    pc = ps = 0.0
    with ClockSampler(0) as clk_p:
        for sc in scenes:
            t0 = time.perf_counter()
            e = nbc.Engine([sc], **opts)
            t1 = time.perf_counter()
            e.step(args.steps)
            e.sync()
            ps += time.perf_counter() - t1
            pc += t1 - t0
            e.close()
    work = n_sub * args.steps
    arm = lambda c, st: {"create_s": c, "step_s": st, "scenes_per_s": args.scenes / (c + st),
                         "subsphere_steps_per_s": work / st}
    # the FP64 oracle on the first scene: its first step against the batched
    # engine's export step from the same state, and its speed
    ex = nbc.Engine([scenes[0]], precision=args.precision, use_graph=False)
    ex.step_export(1)
    first = {"pairs": ex.pairs(), "fcn": ex.pair_forces()}
    ex.close()
    cpu = None if args.no_cpu_baseline else cpu_baseline(args, scenes[0], first)
    line = {"metric": "scenes/s and subsphere-steps/s, batched vs plain (cfg3)",
            "workload": f"cfg3: {args.scenes} settling scenes, clumps log-uniform in [500, 50000], {args.steps} steps each",
            "subspheres_total": n_sub, "batched": arm(bc, bs), "plain": arm(pc, ps), "autotuned_batch": tuned,
            "speedup_steps": ps / bs, "speedup_scenes_per_s": (pc + ps) / (bc + bs),
            "scene0_after": {"mean_height_m": float(last["pos"][:, 2].mean()),
                             "mean_speed_m_s": float(np.linalg.norm(last["vel"], axis=1).mean())},
            "cpu_baseline_scene0": cpu,
            "clocks": {"batched": clk_b.summary(), "plain": clk_p.summary()},
            "dtype": "f32 contact law, f64 positions/quaternions" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded numpy beds)"}
    print(json.dumps(line), flush=True)


def serve_requests(args):
    """The cfg4 requests: (arrival time, scene, steps) in arrival order, and
    the bank bed sizes."""
    import nbc
    rng = np.random.default_rng(20260828)
    sizes = np.unique(np.round(np.exp(np.linspace(np.log(1000), np.log(200_000), args.bank))).astype(int))
    bank = []
    for i, n in enumerate(sizes):
        half = 0.5 * (n * 3.0e-7) ** (1 / 3) + 0.01
        bed = nbc.with_levels(sg.make_poly_bed(int(n), 20260828 + i, half))
        e = nbc.Engine([bed], precision=args.precision)
        e.step(args.settle)
        bank.append(e.restart_scene(bed))
        e.close()
    reqs = []
    t_arr = np.cumsum(rng.exponential(1.0 / args.rate, args.requests))
    for k in range(args.requests):
        n = np.exp(rng.uniform(np.log(1000), np.log(200_000)))
        bed = bank[int(np.argmin(np.abs(np.log(sizes) - np.log(n))))]
        r_i, v, mu = rng.uniform(5e-3, 20e-3), rng.uniform(0.05, 0.5), rng.uniform(0.2, 0.8)
        sc = sg.with_sphere_intruder(bed, r_i, v, mu=mu, surface=98)
        nsteps = int(math.ceil(args.depth_ratio * r_i / (v * sc["params"]["StepSize"])))
        reqs.append((t_arr[k], sc, nsteps))
    return sizes, reqs


def run_cfg2(args):
    """cfg2: the polydisperse penetration bed, 1,000,000 subspheres in clumps
    of 1..8 (radii log-uniform in [0.5, 5] mm, hierarchical grid from the
    level chooser) seeded in layers in a 0.4 x 0.4 m cube wall and settled
    under gravity for at least --settle2 steps and on, 25,000 at a time,
    while some clump still moves faster than 0.5 m/s (at most
    --settle2-max); then a 20 mm sphere intruder, placed
    touching the highest subsphere beneath it, driven down at 0.1 m/s for
    0.5 s.  Reports the force-depth curve (reaction on the intruder against
    the travel of its lowest point since first contact), the bed's state
    after settling and the engine's speed in both phases."""
    import nbc
    bed = nbc.with_levels(sg.make_cfg2())
    N = int(bed["params"]["NumberBody"])
    if args.profile_window is not None:
        # for a launch list: settle --profile-window steps, then restart the
        # state in an eager engine (kernel nodes of a graph with a conditional
        # node are not profiled) and put the profiler range around --steps steps
        import torch
        e = nbc.Engine([bed], precision=args.precision, search_lanes=args.search_lanes)
        e.step(args.profile_window)
        state = e.restart_scene(bed)
        e.close()
        e = nbc.Engine([state], precision=args.precision, use_graph=False, search_lanes=args.search_lanes)
        e.step(3)
        e.sync()
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        e.step(args.steps)
        e.sync()
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        st = e.stats()
        print(json.dumps({"profile_run": True, "subspheres": N, "window": [args.profile_window, args.steps],
                          "rebuilds": st["rebuilds"], "pairs": st["npairs"]}), flush=True)
        e.close()
        return
    e = nbc.Engine([bed], precision=args.precision, search_lanes=args.search_lanes)
    t0 = time.perf_counter()
    e.step(args.settle2)
    e.sync()
    settled_steps = args.settle2
    cl = e.clumps()
    speed = np.linalg.norm(cl["vel"], axis=1)
    # the seeded layers of the full bed reach metres: settle on in chunks
    # until no clump is still falling fast (or the cap)
    while speed.max() > 0.5 and settled_steps < args.settle2_max:
        e.step(25_000)
        e.sync()
        settled_steps += 25_000
        cl = e.clumps()
        speed = np.linalg.norm(cl["vel"], axis=1)
    settle_s = time.perf_counter() - t0
    st = e.stats()
    settled = e.restart_scene(bed)
    top = float((settled["sub"]["pos"][:, 2] + settled["sub"]["radius"]).max())
    rmax = float(settled["sub"]["radius"].max())
    cube = settled["cube"]
    lo = cube["centre"] - cube["half"] + 3 * rmax
    hi = np.array(cube["centre"] + cube["half"] - 3 * rmax)
    hi[2] = top - 3 * rmax
    phi = bulk_packing_fraction(settled["sub"]["pos"], settled["sub"]["radius"], lo, hi)
    e.close()
    sc = sg.with_sphere_intruder(settled, 0.02, 0.1, surface=98)
    dt = float(sc["params"]["StepSize"])
    total = int(round(0.5 / dt))
    nchunk = 100
    e = nbc.Engine([sc], precision=args.precision, search_lanes=args.search_lanes)
    z0 = float(sc["intruder"]["pos"][2])
    curve, done = [[0.0, 0.0, 0.0, 0.0]], 0
    t0 = time.perf_counter()
    for c in range(nchunk):
        n = (total * (c + 1)) // nchunk - done
        e.step(n)
        done += n
        it = e.intruder()
        curve.append([done * dt, z0 - float(it["pos"][2])] + [float(v) for v in it["reaction"][1:]])
    e.sync()
    pen_s = time.perf_counter() - t0
    st2 = e.stats()
    e.close()
    line = {"metric": "force-depth curve and subsphere-steps/s (cfg2)",
            "workload": f"cfg2: {N} subspheres, settled {settled_steps} steps, 20 mm sphere intruder at 0.1 m/s for 0.5 s "
                        f"({total} steps of {dt:.3e} s)",
            "settle": {"steps": settled_steps, "seconds": settle_s, "subsphere_steps_per_s": N * settled_steps / settle_s,
                       "rule": f"at least {args.settle2} steps, then 25,000 at a time while some clump moves faster "
                               f"than 0.5 m/s, at most {args.settle2_max}",
                       "rebuilds": st["rebuilds"], "pairs": st["npairs"], "bed_top_m": top,
                       "bulk_packing_fraction": phi,
                       "bulk_region": "at least 3 r_max from every wall and below the bed top (seeded Monte Carlo)",
                       "clump_speed_mean": float(speed.mean()), "clump_speed_max": float(speed.max())},
            "penetration": {"steps": total, "seconds": pen_s, "subsphere_steps_per_s": N * total / pen_s,
                            "rebuilds": st2["rebuilds"], "pairs": st2["npairs"], "err": st2["err"]},
            "curve_columns": ["t_s", "depth_m", "reaction_y_N", "reaction_z_N"],
            "curve": curve,
            "dtype": "f32 contact law, f64 positions/quaternions" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded numpy bed settled by the engine)"}
    print(json.dumps(line), flush=True)


def bulk_packing_fraction(pos, radius, lo, hi, n=100_000, seed=3):
    """Solid fraction of the box [lo, hi] by seeded Monte Carlo: a point is
    solid when some sphere contains it (neighbours within the largest radius
    from a k-d tree)."""
    from scipy.spatial import cKDTree
    pts = np.random.default_rng(seed).uniform(lo, hi, (n, 3))
    tree = cKDTree(pos)
    rmax = float(radius.max())
    inside = np.zeros(n, dtype=bool)
    for k, cand in enumerate(tree.query_ball_point(pts, rmax)):
        if cand:
            c = np.asarray(cand)
            inside[k] = bool((((pos[c] - pts[k]) ** 2).sum(1) <= radius[c] ** 2).any())
    return float(inside.mean())


def run_serve(args):
    """cfg4: a Poisson stream (rate --rate) of --requests penetration
    requests.  Beds come from a bank of pre-settled polydisperse beds (clumps
    of 1..8 subspheres, radii log-uniform in [0.5, 5] mm) at log-spaced sizes
    between 1k and 200k subspheres; a request takes the bank bed nearest its
    size (log-uniform in [1k, 200k]), a sphere intruder of radius U[5, 20] mm
    driven down at U[0.05, 0.5] m/s, friction U[0.2, 0.8], and ends when the
    intruder has travelled --depth-ratio x its radius.  Served: nbc_server
    (admission by HBM budget, continuous batching); plain: the same requests
    solved one at a time, their time-to-result from the same arrival times."""
    import nbc
    sizes, reqs = serve_requests(args)
    work = sum(int(sc["params"]["NumberBody"]) * n for _, sc, n in reqs)
    # served: arrivals replayed in real time
    srv = nbc.Server(budget_bytes=args.budget_gb * 1e9, max_active=args.slots, cohort=args.cohort,
                     precision=args.precision)
    t0 = time.perf_counter()
    nxt, ids, done_at, failed = 0, {}, {}, []
    while len(done_at) < len(reqs):
        now = time.perf_counter() - t0
        while nxt < len(reqs) and reqs[nxt][0] <= now:
            ids[srv.submit(reqs[nxt][1], reqs[nxt][2], 100)] = nxt
            nxt += 1
        st = srv.advance(chunk=args.chunk)
        if st["running"] == 0 and st["queued"] == 0 and nxt < len(reqs):
            time.sleep(max(0.0, reqs[nxt][0] - (time.perf_counter() - t0)))
        now = time.perf_counter() - t0
        for rid in [r for r in ids if srv.state(r)[0] >= 2]:
            k = ids.pop(rid)
            done_at[k] = now
            try:
                srv.result(rid)
            except nbc.NbcError as err:
                failed.append({"request": k, "subspheres": int(reqs[k][1]["params"]["NumberBody"]),
                               "intruder_radius": reqs[k][1]["intruder"]["radius"],
                               "speed": -float(reqs[k][1]["intruder"]["vel"][2]),
                               "friction": reqs[k][1]["params"]["Frcoe"], "error": str(err)})
            srv.release(rid)
    makespan = time.perf_counter() - t0
    srv.close()
    ttr_srv = [done_at[k] - reqs[k][0] for k in range(len(reqs))]
    # plain: the same requests one at a time; time-to-result from the same arrivals
    svc, failed_plain = [], []
    for k, (_, sc, n) in enumerate(reqs):
        t = time.perf_counter()
        e = nbc.Engine([sc], precision=args.precision, pair_slack=1.6)
        try:
            e.step(n)
            e.sync()
            e.intruder_history(count=min(n, 1024))
        except nbc.NbcError:
            failed_plain.append(k)
        e.close()
        svc.append(time.perf_counter() - t)
    fin, ttr_plain = 0.0, []
    for (arr, _, _), sv in zip(reqs, svc):
        fin = max(arr, fin) + sv
        ttr_plain.append(fin - arr)
    q = lambda v, p: float(np.percentile(v, p))
    # the error of a served result against FP64: the first request's first
    # step against the oracle from the same state (pair list and per-contact
    # normal force), and the oracle's speed on it
    ex = nbc.Engine([reqs[0][1]], precision=args.precision, use_graph=False)
    ex.step_export(1)
    first = {"pairs": ex.pairs(), "fcn": ex.pair_forces()}
    ex.close()
    cpu = None if args.no_cpu_baseline else cpu_baseline(args, reqs[0][1], first)
    line = {"metric": "time-to-result p50/p99 and throughput, served vs plain (cfg4)",
            "workload": f"cfg4: {len(reqs)} penetration requests, Poisson rate {args.rate}/s, "
                        f"subspheres log-uniform in [1k, 200k] (bank of {len(sizes)} pre-settled beds), "
                        f"depth {args.depth_ratio} x intruder radius",
            "subsphere_steps_total": work,
            "served": {"p50_s": q(ttr_srv, 50), "p99_s": q(ttr_srv, 99), "makespan_s": makespan,
                       "requests_per_s": len(reqs) / makespan, "subsphere_steps_per_s": work / makespan},
            "plain": {"p50_s": q(ttr_plain, 50), "p99_s": q(ttr_plain, 99), "makespan_s": fin,
                      "requests_per_s": len(reqs) / sum(svc), "subsphere_steps_per_s": work / sum(svc)},
            "throughput_ratio": (work / makespan) / (work / sum(svc)),
            "failed": failed, "failed_plain": failed_plain,
            "slots": args.slots, "cohort": args.cohort, "budget_gb": args.budget_gb,
            "request0_vs_fp64": cpu,
            "dtype": "f32 contact law, f64 positions/quaternions" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded numpy beds settled by the engine)"}
    print(json.dumps(line), flush=True)


def run_reference(args, world, rank, local):
    """The reference arm: the reference's clump step restated in C (oracle/,
    FP64, OpenMP over every host thread; the reference itself is a GPU
    program with no CPU implementation), on the same workload and start
    state, each step of a sample bounded to a few minutes.  It loads nothing
    of the engine."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    scene, config = workload(args)
    N = config["subspheres"]
    o = oracle.OracleScene(scene, threads=threads)
    t = time.perf_counter()
    o.step(max(1, args.warmup))
    warm = (time.perf_counter() - t) / max(1, args.warmup)
    budget = 150.0
    steps = max(1, min(args.steps, int(budget / max(warm, 1e-6))))
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    v = N * steps / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "subsphere-steps/s",
        "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded numpy bed settled by the engine, no dataset)",
        "config": config,
        "engine": {"implementation": "CPU restatement of the reference clump step (oracle/), FP64, OpenMP"},
        "cpu_baseline": {"value": v, "unit": "subsphere-steps/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} steps of the {N}-subsphere scene after {max(1, args.warmup)} warm-up "
                                   "steps from the same start state"},
        "e2e": {"value": v, "unit": "subsphere-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=19990)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "f64"])
    ap.add_argument("--clumps", type=int, default=50_000, help="with --from-seed: clumps of the cfg1 bed")
    ap.add_argument("--from-seed", action="store_true", help="start from the seeded (falling) cfg1 bed")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--graph", type=int, default=1, help="1: CUDA graphs; 0: eager launches (for ncu)")
    ap.add_argument("--autotune", type=int, default=1, help="1: launch shapes from nbc_autotune (untimed)")
    ap.add_argument("--batch-scenes", type=int, default=64, help="batched record: cfg3 scenes (0: skip)")
    ap.add_argument("--batch-settle", type=int, default=2000, help="batched record: settling steps (untimed)")
    ap.add_argument("--batch-steps", type=int, default=300, help="batched record: timed steps")
    ap.add_argument("--profile", action="store_true",
                    help="short run for profilers: warm-up + timed steps only, no e2e / CPU legs")
    ap.add_argument("--pair-slack", type=float, default=0.0,
                    help="pair buffer capacity over the first list (0 = engine default)")
    ap.add_argument("--search-lanes", type=int, default=0, help="lanes per subsphere in the neighbour search")
    ap.add_argument("--scene", default=None, help="run this scene file instead of generating cfg1")
    ap.add_argument("--save-state", default=None, help="advance --advance steps, save the state to this file, exit")
    ap.add_argument("--advance", type=int, default=18000)
    ap.add_argument("--workload", default="cfg1", choices=["cfg1", "cfg2", "cfg3", "cfg4"])
    ap.add_argument("--settle2", type=int, default=150_000, help="cfg2: settling steps of the bed")
    ap.add_argument("--settle2-max", type=int, default=325_000, help="cfg2: most settling steps (settles on while a clump moves faster than 0.5 m/s)")
    ap.add_argument("--scenes", type=int, default=256, help="cfg3: number of scenes")
    ap.add_argument("--profile-window", type=int, default=None,
                    help="cfg2/cfg3: eager run for a profiler range of --steps steps after this many")
    ap.add_argument("--requests", type=int, default=200, help="cfg4: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="cfg4: mean arrivals per second")
    ap.add_argument("--bank", type=int, default=8, help="cfg4: pre-settled beds in the bank")
    ap.add_argument("--settle", type=int, default=3000, help="cfg4: settling steps of each bank bed")
    ap.add_argument("--depth-ratio", type=float, default=0.5, help="cfg4: intruder travel / radius")
    ap.add_argument("--slots", type=int, default=64, help="cfg4: requests running at once at most")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="cfg4: device memory for requests")
    ap.add_argument("--chunk", type=int, default=256, help="cfg4: steps per server round")
    ap.add_argument("--cohort", type=int, default=1, help="cfg4: requests per server cohort (shared engine) at most")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup(args)
    if args.workload == "cfg2":
        run_cfg2(args)
    elif args.workload == "cfg3":
        run_batch(args)
    elif args.workload == "cfg4":
        run_serve(args)
    elif args.save_state:
        save_state(args)
    elif args.impl == "reference":
        run_reference(args, world, rank, local)
    else:
        run_b200(args, world, rank, local)


if __name__ == "__main__":
    main()
