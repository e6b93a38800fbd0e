"""Benchmark: plain DeepWalk on a dynamic R-MAT graph (scale 20, ~16M edges,
log-uniform weights in [1, 2^20)). One step = one update batch of 100K edges
(50K absent-pair inserts + 50K uniform deletes) followed by 1M DeepWalk walks
of length 80 (one per vertex), one launch per job.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `value` = walk steps per second over the whole
device-timed step (updates included), inputs resident in HBM; `e2e` = the same
metric through the C ABI with pinned host buffers (batches copied in, every
walk row copied out, inside the timed region). With N > 1 (torchrun) every
rank runs a full replica (weak scaling, no collective on the data path).

At N = 1 the default run also measures, each in a child process with its own
clock record, the node2vec workload (R-MAT 22), the batched form against the
plain form (256 mixed jobs on R-MAT 22), the served form against the plain
form (Poisson requests on R-MAT 24) and the reference's own CUDA build on the
DeepWalk workload with weights below 2^16, and reports them under
`other_workloads` (`--no-extras` skips them; they never run under a
profiler).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR = 20, 16
W_LO, W_HI = 1, 1 << 20
WALK_LEN = 80
BATCH_INS, BATCH_DEL = 50_000, 50_000
GRAPH_SEED = 1234 + 2
BYTES_PER_STEP = 32  # algorithmic bytes per produced walk step (vertex 8, alias 8, member 4+4, group 4, store 4)
WORKLOAD = "plain-deepwalk-rmat20"


def headline_config(m: int, world: int) -> dict:
    """The config block both arms print for the DeepWalk workload."""
    return {"workload": WORKLOAD, "scale": SCALE, "edge_factor": EDGE_FACTOR, "m": int(m),
            "weights": "loguniform[1,2^20)", "walks": 1 << SCALE, "walk_len": WALK_LEN,
            "batch": {"insert": BATCH_INS, "delete": BATCH_DEL}, "form": "plain (one launch per job)",
            "l2": "inputs larger than L2 (graph state and 320 MB walk output per step)",
            "clocks": "nvidia-smi samples from warm-up to the end of the e2e timed region",
            "parallelism": f"replicas x{world}"}


def make_workload(steps_total: int, w_hi: int = W_HI):
    from bingo_b200 import gen
    n = 1 << SCALE
    src, dst = gen.rmat(SCALE, EDGE_FACTOR, seed=GRAPH_SEED)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, W_LO, w_hi, seed=GRAPH_SEED + 1)
    ug = gen.UpdateGen(n, src, dst, seed=GRAPH_SEED + 2)
    batches = []
    for _ in range(steps_total):
        ins = ug.inserts(BATCH_INS, gen.W_LOGUNIFORM, W_LO, w_hi)
        dels = ug.deletes(BATCH_DEL)
        batches.append((ins, dels))
    return n, src, dst, w, batches


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per produced step
# of k_walk<DEEPWALK> on this workload, from one ncu capture of one launch:
# the 4th walk launch of `bench.py --steps 3 --warmup 3` (the first timed
# step, 31,776,603 produced steps; 2.796 GB read + 0.334 GB written).
# roofline.traffic scales it to the live run's steps per launch.
WALK_DRAM_BYTES_PER_STEP = 98.5
WALK_DRAM_SOURCE = ("ncu capture of one k_walk<DEEPWALK> launch (4th launch, 31,776,603 steps) of "
                    "bench.py --steps 3 --warmup 3, scaled to this run's steps per launch")


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"bingo_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self, t0: float, t1: float):
        """Samples whose timestamp lies in the host-time window [t0, t1]."""
        if not self.proc:
            return None
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.close()
        import datetime
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                if not (t0 - 0.05 <= ts <= t1 + 0.05):
                    continue
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reduce_max(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# --------------------------------------------------------------------------- CPU leg
CPU_WALK_FORM = "OpenMP over all host threads, 16 walks per thread in flight"


def scaled_note(walks, n):
    return "" if walks >= n else f", walk time scaled to {n} walks"


class CpuRun:
    """The CPU oracle (OpenMP, all host threads) on the same graph: load once,
    then per step one full update batch and a bounded walk sample."""

    def __init__(self, n, src, dst, w):
        from oracle import pyoracle as po
        self.n = n
        self.ex = po.ExactGraph(n)
        self.ex.load(src, dst, w)

    def step(self, batch, walks: int, seed: int, app: int = 0, length: int = WALK_LEN, p: float = 0.5,
             q: float = 2.0):
        ins, dels = batch
        t0 = time.perf_counter()
        self.ex.insert(*ins)
        self.ex.delete(*dels)
        t_upd = time.perf_counter() - t0
        rng = np.random.default_rng(seed)
        starts = np.sort(rng.choice(self.n, size=walks, replace=False)).astype(np.uint32)
        t0 = time.perf_counter()
        if app in (0, 2):  # DeepWalk / PPR: several walks per thread in flight, the same rows as walk()
            rows = self.ex.walk_interleaved(app, length, starts, seed=seed, job_id=0)
        else:
            rows = self.ex.walk(app, length, starts, seed=seed, job_id=0, p=p, q=q)
        t_walk = time.perf_counter() - t0
        steps = int((rows >= 0).sum() - len(starts))
        scale = self.n / walks  # extrapolate the walk sample to one walk per vertex
        value = steps * scale / (t_upd + t_walk * scale)
        return dict(value=value, ms_per_step=(t_upd + t_walk * scale) * 1e3, t_update=t_upd, t_walk=t_walk,
                    walk_steps=steps, walks=walks,
                    walk_steps_per_s=steps / t_walk, edge_updates_per_s=(len(ins[0]) + len(dels[0])) / t_upd)


def run_reference(args):
    """The reference arm: the reference has no CPU implementation of the path,
    so the CPU oracle port (OpenMP, all host threads) stands in for it, on the
    same graph and batches; each step is one full update batch plus a bounded
    walk sample, extrapolated to the full step."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    # Inputs from the generators linked into the oracle library: this arm
    # never maps the engine library (libbingo.so).
    from bingo_b200 import gen
    from oracle import pyoracle as po
    gen.bind(po.gen_lib())
    n, src, dst, w, batches = make_workload(args.warmup + args.steps)
    walks = min(args.ref_walks, n)
    vals, ms, last = [], [], None
    cpu = CpuRun(n, src, dst, w)
    for i in range(args.warmup + args.steps):
        r = cpu.step(batches[i], walks, seed=100 + i)
        if i >= args.warmup:
            vals.append(r["value"])
            ms.append(r["ms_per_step"])
            last = r
    value = float(np.mean(vals))
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": "walk_steps_per_s", "value": value, "unit": "steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(ms)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": headline_config(len(src), world),
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cores, "kind": "port",
                         "sample": f"per step: one full 50K+50K update batch + {walks} walks x {WALK_LEN} "
                                   f"(oracle port, {CPU_WALK_FORM})" + scaled_note(walks, n)},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "walk_steps_per_s": last["walk_steps_per_s"], "edge_updates_per_s": last["edge_updates_per_s"],
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- batched: 256 mixed jobs on R-MAT 22
B_SCALE, B_PHASES, B_JOBS_PER_PHASE = 22, 16, 16
B_SEED = 1234 + 4


def make_batched_workload(steps_total: int):
    """R-MAT scale 22, uniform [1, 65535] weights; 256 jobs (16 phases x 16)
    with log-uniform start counts in [1K, 1M], lengths uniform in [5, 200],
    apps uniform over {DeepWalk, node2vec with p, q in {0.25, 1, 4}, PPR
    stop 0.15}; after each phase an update chunk of log-uniform [1K, 1M]
    edges, half absent-pair inserts and half uniform deletes. Chunk sizes are
    fixed across steps; their contents are fresh every step."""
    from bingo_b200 import DEEPWALK, NODE2VEC, PPR, gen
    n = 1 << B_SCALE
    src, dst = gen.rmat(B_SCALE, EDGE_FACTOR, seed=B_SEED)
    w = gen.weights(len(src), gen.W_UNIFORM, 1, 65535, seed=B_SEED + 1)
    rng = np.random.default_rng(B_SEED + 2)
    deg = np.bincount(src, minlength=n)
    walkable = np.nonzero(deg)[0].astype(np.uint32)
    pq = [(p_, q_) for p_ in (0.25, 1.0, 4.0) for q_ in (0.25, 1.0, 4.0)]
    jobs = []
    for j in range(B_PHASES * B_JOBS_PER_PHASE):
        k = int(np.exp(rng.uniform(np.log(1e3), np.log(1e6))))
        L = int(rng.integers(5, 201))
        app = int(rng.integers(0, 3))
        p_, q_ = pq[int(rng.integers(0, 9))]
        jobs.append(dict(app=[DEEPWALK, NODE2VEC, PPR][app], length=L, starts=rng.choice(walkable, size=k),
                         p=p_, q=q_, stop_prob=0.15, job_id=j))
    chunk = [int(np.exp(rng.uniform(np.log(1e3), np.log(1e6)))) for _ in range(B_PHASES)]
    ug = gen.UpdateGen(n, src, dst, seed=B_SEED + 3)
    steps = []
    for _ in range(steps_total):
        ph = []
        for c in chunk:
            ph.append((ug.inserts(c // 2, gen.W_UNIFORM, 1, 65535), ug.deletes(c - c // 2)))
        steps.append(ph)
    return n, src, dst, w, jobs, chunk, steps


def run_batched(args):
    import torch
    from bingo_b200 import Graph, WalkJob
    world, rank, local = dist_setup()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    total = args.warmup + args.steps
    n, src, dst, w, jobs, chunk, steps = make_batched_workload(total)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)  # noqa: E731
    starts = [t(j["starts"]) for j in jobs]
    outs = [torch.empty((len(j["starts"]), j["length"]), dtype=torch.int32, device=dev) for j in jobs]
    # fixed device batch buffers per chunk, refilled each step from per-step copies
    buf = [((t(ins[0]), t(ins[1]), t(ins[2])), (t(de[0]), t(de[1]))) for ins, de in steps[0]]
    per_step = [[((t(i[0]), t(i[1]), t(i[2])), (t(d[0]), t(d[1]))) for i, d in ph] for ph in steps]
    slots = [torch.empty(len(steps[0][c][0][0]), dtype=torch.int32, device=dev) for c in range(B_PHASES)]

    def walkjobs(phase, seed):
        js = []
        for j in range(phase * B_JOBS_PER_PHASE, (phase + 1) * B_JOBS_PER_PHASE):
            J = jobs[j]
            js.append(WalkJob(app=J["app"], length=J["length"], starts=starts[j], n_starts=len(J["starts"]),
                              job_id=J["job_id"], seed=seed, p=J["p"], q=J["q"], stop_prob=J["stop_prob"],
                              out=outs[j]))
        return js

    def refill(step):
        for c in range(B_PHASES):
            for dstb, srcb in zip(buf[c][0] + buf[c][1], per_step[step][c][0] + per_step[step][c][1]):
                dstb.copy_(srcb, non_blocking=True)

    tune_report = {}

    def time_form(form):
        g = Graph(device=local, synchronous=(form == "plain"))
        g.set_stream(stream.cuda_stream)
        g.load_edges(src, dst, w, n)
        g.sync()
        if form == "batched":
            # Autotune on one phase's jobs and an update sample of the first
            # phase's inserts followed by the largest phase's, then the first
            # phase's deletes (their slots are valid once the first inserts are
            # in); the sample is undone, so the timed steps start from the
            # loaded graph.
            refill(0)
            big = int(np.argmax(chunk))
            ins = tuple(torch.cat([x0, xb]) for x0, xb in zip(buf[0][0], buf[big][0]))
            tune_report.update(g.autotune(walkjobs(0, seed=999), inserts=ins, deletes=buf[0][1], repeats=2))
        e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(total)]
        steps0 = None
        for i in range(total):
            if i == args.warmup:
                g.sync()
                torch.cuda.synchronize(dev)
                steps0 = g.stats()["walk_steps"]
            e[i][0].record(stream)
            refill(i)
            if form == "plain":
                for ph in range(B_PHASES):
                    for job in walkjobs(ph, seed=1000 + i):
                        g.walk_jobs([job], mode=1)
                    (a, b, c), (du, ds) = buf[ph]
                    g.insert_batch(a, b, c, out_slots=slots[ph])
                    g.delete_batch(du, ds)
            else:
                ops = []
                for ph in range(B_PHASES):
                    (a, b, c), (du, ds) = buf[ph]
                    ops += [("walk", walkjobs(ph, seed=1000 + i)), ("insert", a, b, c, slots[ph]), ("delete", du, ds)]
                g.run(ops, graph=True)
            e[i][1].record(stream)
        g.sync()
        torch.cuda.synchronize(dev)
        wsteps = g.stats()["walk_steps"] - steps0
        ms = sum(e[i][0].elapsed_time(e[i][1]) for i in range(args.warmup, total))
        g.close()
        upd = sum(chunk) * args.steps
        return {"walk_steps_per_s": wsteps / (ms / 1e3), "ms_per_step": ms / args.steps,
                "edge_updates_per_s": upd / (ms / 1e3), "walk_steps_per_step": wsteps / args.steps}

    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t_busy0 = time.time()
    plain = time_form("plain")
    default = time_form("batched-default")
    batched = time_form("batched")
    clk = clocks.stop(t_busy0, time.time())
    if rank == 0:
        line = {"metric": "walk_steps_per_s", "value": batched["walk_steps_per_s"], "unit": "steps/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batched["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic",
                "config": {"workload": f"batched-rmat{B_SCALE}", "scale": B_SCALE, "m": int(len(src)),
                           "weights": "uniform[1,65535]", "jobs": len(jobs), "phases": B_PHASES,
                           "walks_per_step": int(sum(len(j["starts"]) for j in jobs)),
                           "update_edges_per_step": int(sum(chunk)),
                           "form": "one CUDA graph per step: 16 x (16-job persistent walk launch, insert, delete)",
                           "knobs": "autotuned (bingo_autotune) before the timed steps"},
                "batched": batched, "plain": plain, "batched_default_knobs": default, "autotune": tune_report,
                "batched_over_plain": batched["walk_steps_per_s"] / plain["walk_steps_per_s"], "clocks": clk}
        print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- served: Poisson requests on R-MAT 24
S_SEED = 1234 + 5


def make_trace(rng, n, walkable, ug, n_req, rate, p_update):
    """Poisson arrivals at `rate` requests/s. A request is an update batch
    (probability p_update; log-uniform 1..1M edges; insert or delete with
    equal odds) or a walk query (log-uniform 1..100K starts over vertices with
    out-edges, length 80, DeepWalk or PPR with stop 0.15)."""
    from bingo_b200 import DEEPWALK, PPR, gen
    t = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    reqs = []
    for i in range(n_req):
        if rng.random() < p_update:
            k = int(np.exp(rng.uniform(0, np.log(1e6))))
            if rng.random() < 0.5:
                reqs.append(("insert", t[i], ug.inserts(k, gen.W_LOGUNIFORM, 1, 2 ** 32 - 1)))
            else:
                reqs.append(("delete", t[i], ug.deletes(k)))
        else:
            k = int(np.exp(rng.uniform(0, np.log(1e5))))
            app = DEEPWALK if rng.random() < 0.5 else PPR
            reqs.append(("walk", t[i], (app, rng.choice(walkable, size=k).astype(np.uint32), i)))
    return reqs


def pct(xs, q):
    return float(np.percentile(np.asarray(xs, np.float64), q)) if len(xs) else None


def run_served(args):
    import torch
    from bingo_b200 import DEEPWALK, Graph, gen
    world, rank, local = dist_setup()
    if rank != 0:
        return
    scale = args.served_scale
    n = 1 << scale
    src, dst = gen.rmat(scale, EDGE_FACTOR, seed=S_SEED)
    w = gen.weights(len(src), gen.W_LOGUNIFORM, 1, 2 ** 32 - 1, seed=S_SEED + 1)
    walkable = np.nonzero(np.bincount(src, minlength=n))[0].astype(np.uint32)
    ug = gen.UpdateGen(n, src, dst, seed=S_SEED + 2)
    rng = np.random.default_rng(S_SEED + 3)
    rates = [float(x) for x in args.rates.split(",")]
    traces = [make_trace(rng, n, walkable, ug, args.requests, r, args.p_update) for r in rates]
    g = Graph(device=local, node2vec=False, arena_factor=1.25)

    def prepare(upto):
        """Base graph plus the update batches of every earlier trace, then one
        untimed walk (first-use and buffer-growth costs stay out of both arms)."""
        g.load_edges(src, dst, w, n)
        for tr in traces[:upto]:
            for kind, _, x in tr:
                if kind == "insert":
                    g.insert_batch(*x, return_slots=False)
                elif kind == "delete":
                    g.delete_batch(*x)
        # The largest query a trace can hold, so that neither arm grows its
        # staging buffers inside its timed region.
        g.walk(app=DEEPWALK, length=WALK_LEN, starts=np.resize(walkable, 100_000), seed=1, job_id=1 << 30)
        g.sync()

    def outputs(tr):
        tot = sum(len(x[1]) * WALK_LEN for kind, _, x in tr if kind == "walk")
        pool = torch.empty(max(tot, 1), dtype=torch.int32).pin_memory()
        outs, off = [], 0
        for kind, _, x in tr:
            if kind == "walk":
                k = len(x[1])
                outs.append(pool[off:off + k * WALK_LEN].view(k, WALK_LEN))
                off += k * WALK_LEN
            else:
                outs.append(None)
        return outs

    # Untimed warm-up of both forms (module loads, first allocations, update
    # scratch), on a copy of the graph that each rate reloads anyway.
    prepare(0)
    wu = make_trace(np.random.default_rng(S_SEED + 9), n, walkable, gen.UpdateGen(n, src, dst, seed=S_SEED + 8),
                    24, 1000.0, 0.25)
    wouts = outputs(wu)
    g.serve_start(output_budget_bytes=args.serve_budget << 20, max_update_batch=1 << 20, idle_timeout_us=3000)
    wt = [g.submit_walk(app=x[0], length=WALK_LEN, starts=x[1], seed=7, job_id=x[2], stop_prob=0.15, out=o)[0]
          if k == "walk" else g.submit_update(k, *x)[0] for (k, _, x), o in zip(wu, wouts)]
    for t in wt:
        g.serve_wait(t, timeout_us=600_000_000)
    g.serve_stop()
    prepare(0)
    for (k, _, x), o in zip(wu, wouts):
        if k == "walk":
            g.walk(app=x[0], length=WALK_LEN, starts=x[1], seed=7, job_id=x[2], stop_prob=0.15, out=o)
        elif k == "insert":
            g.insert_batch(*x, return_slots=False)
        else:
            g.delete_batch(*x)

    results = []
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t_busy0 = time.time()
    for ri, (rate, tr) in enumerate(zip(rates, traces)):
        outs = outputs(tr)
        # ---- served: continuous batching
        prepare(ri)
        s0 = g.stats()["walk_steps"]
        g.serve_start(output_budget_bytes=args.serve_budget << 20, max_update_batch=1 << 20, idle_timeout_us=3000)
        gc.collect()
        gc.disable()  # no collector pauses inside either arm's timed region
        t0 = time.monotonic_ns()
        tickets = []
        for (kind, at, x), out in zip(tr, outs):
            due = t0 + int(at * 1e9)
            while time.monotonic_ns() < due:
                pass
            if kind == "walk":
                app, starts, jid = x
                tickets.append((kind, due, g.submit_walk(app=app, length=WALK_LEN, starts=starts, seed=7,
                                                         job_id=jid, stop_prob=0.15, out=out)[0]))
            else:
                tickets.append((kind, due, g.submit_update(kind, *x)[0]))
        lat = {"walk": [], "update": []}
        last_ready = t0
        for kind, due, t in tickets:
            st = g.serve_wait(t, timeout_us=600_000_000)
            assert st["status"] == 0, st
            lat["walk" if kind == "walk" else "update"].append((st["ready_ns"] - due) / 1e6)
            last_ready = max(last_ready, st["ready_ns"])
        gc.enable()
        smet = g.serve_metrics()
        g.serve_stop()
        served_steps = g.stats()["walk_steps"] - s0
        served_span = (last_ready - t0) / 1e9
        # ---- plain: one request at a time in arrival order (a queue, no batching)
        prepare(ri)
        s0 = g.stats()["walk_steps"]
        plat = {"walk": [], "update": []}
        ptrace = []
        gc.collect()
        gc.disable()
        t0 = time.monotonic_ns()
        for (kind, at, x), out in zip(tr, outs):
            due = t0 + int(at * 1e9)
            while time.monotonic_ns() < due:
                pass
            t_call = time.monotonic_ns()
            if kind == "walk":
                app, starts, jid = x
                g.walk(app=app, length=WALK_LEN, starts=starts, seed=7, job_id=jid, stop_prob=0.15, out=out)
            elif kind == "insert":
                g.insert_batch(*x, return_slots=False)
            else:
                g.delete_batch(*x)
            plat["walk" if kind == "walk" else "update"].append((time.monotonic_ns() - due) / 1e6)
            ptrace.append((kind, len(x[1]) if kind == "walk" else len(x[0]), round((time.monotonic_ns() - due) / 1e6, 3),
                           round((time.monotonic_ns() - t_call) / 1e6, 3)))
        plain_span = (time.monotonic_ns() - t0) / 1e9
        gc.enable()
        plain_steps = g.stats()["walk_steps"] - s0
        n_walk = len(lat["walk"])
        upd_edges = sum(len(x[0]) for kind, _, x in tr if kind != "walk")
        results.append({
            "rate_req_s": rate, "requests": len(tr), "walk_queries": n_walk, "update_batches": len(tr) - n_walk,
            "update_edges": upd_edges,
            "served": {"walk_p50_ms": pct(lat["walk"], 50), "walk_p99_ms": pct(lat["walk"], 99),
                       "update_p50_ms": pct(lat["update"], 50), "update_p99_ms": pct(lat["update"], 99),
                       "walk_steps_per_s": served_steps / served_span, "requests_per_s": len(tr) / served_span,
                       "span_s": served_span, "scheduler": smet},
            "plain": {"walk_p50_ms": pct(plat["walk"], 50), "walk_p99_ms": pct(plat["walk"], 99),
                      "update_p50_ms": pct(plat["update"], 50), "update_p99_ms": pct(plat["update"], 99),
                      "walk_steps_per_s": plain_steps / plain_span, "requests_per_s": len(tr) / plain_span,
                      "span_s": plain_span, "slowest_requests": sorted(((i,) + t for i, t in enumerate(ptrace)), key=lambda z: -z[4])[:8]},
        })
    clk = clocks.stop(t_busy0, time.time())
    best = max(results, key=lambda r: r["served"]["walk_steps_per_s"])
    line = {"metric": "walk_steps_per_s", "value": best["served"]["walk_steps_per_s"], "unit": "steps/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"served-rmat{scale}", "scale": scale, "m": int(len(src)),
                       "weights": "loguniform[1,2^32)", "p_update": args.p_update, "walk_len": WALK_LEN,
                       "requests_per_rate": args.requests, "serve_budget_mb": args.serve_budget,
                       "latency": "arrival (scheduled) to result in pinned host memory"},
            "sweep": results, "clocks": clk}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- this engine on a given workload
def measure_engine(args, n, src, dst, w, batches, local, app=None, length=WALK_LEN, p=0.5, q=2.0):
    """This engine on the given workload: device-timed steps (inputs in HBM).
    app None = DeepWalk."""
    import torch
    from bingo_b200 import DEEPWALK, NODE2VEC, PLAIN, Graph, WalkJob
    app = DEEPWALK if app is None else app
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    # The node2vec adjacency index only for node2vec, as the reference builds
    # it only for node2vec runs (NODE2VEC = 0 unless the app is node2vec,
    # include/api.h:26, src/apps.cu:14-15).
    g = Graph(device=local, synchronous=False, node2vec=(app == NODE2VEC))
    g.set_stream(stream.cuda_stream)
    g.load_edges(src, dst, w, n)

    def dev_i32(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)

    db = [((dev_i32(i[0]), dev_i32(i[1]), dev_i32(i[2])), (dev_i32(d[0]), dev_i32(d[1]))) for i, d in batches]
    out = torch.empty((n, length), dtype=torch.int32, device=dev)
    slots = torch.empty(max(len(b[0][0]) for b in batches), dtype=torch.int32, device=dev)
    total = args.warmup + args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(total)]
    upd_edges = 0
    for i in range(total):
        if i == args.warmup:
            g.sync()
            s0 = g.stats()
        (a, b, c), (du, ds) = db[i]
        if i >= args.warmup:
            upd_edges += a.numel() + du.numel()
        ev[i][0].record(stream)
        g.insert_batch(a, b, c, out_slots=slots[:a.numel()])
        g.delete_batch(du, ds)
        ev[i][1].record(stream)
        g.walk_jobs([WalkJob(app=app, length=length, n_starts=n, first=0, job_id=i, seed=1, p=p, q=q, out=out)],
                    mode=PLAIN)
        ev[i][2].record(stream)
    g.sync()
    torch.cuda.synchronize(dev)
    s1 = g.stats()
    steps = s1["walk_steps"] - s0["walk_steps"]
    upd = sum(ev[i][0].elapsed_time(ev[i][1]) for i in range(args.warmup, total)) / 1e3
    wlk = sum(ev[i][1].elapsed_time(ev[i][2]) for i in range(args.warmup, total)) / 1e3
    whole = sum(ev[i][0].elapsed_time(ev[i][2]) for i in range(args.warmup, total)) / 1e3
    chk = g.check(raise_on_corrupt=False)  # after the timed steps: the store they left is sound
    g.close()
    if chk["bad_vertices"]:
        raise SystemExit(f"bench: the graph store fails its check after the timed updates: {chk}")
    r = {"value": steps / whole, "walk_steps_per_s": steps / wlk, "edge_updates_per_s": upd_edges / upd,
         "walk_kernel_ms_per_step": wlk * 1e3 / args.steps, "update_ms_per_step": upd * 1e3 / args.steps,
         "steps_per_walk_phase": steps / args.steps,
         "store_check": {"bad_vertices": chk["bad_vertices"], "live_edges": chk["live_edges"]}}
    if app == NODE2VEC:
        trials = s1["walk_trials"] - s0["walk_trials"]
        probes = s1["walk_probes"] - s0["walk_probes"]
        r.update(trials_per_step=trials / max(steps, 1), probes_per_step=probes / max(steps, 1),
                 algorithmic_gbs=(trials * N2V_BYTES_PER_TRIAL + probes * N2V_BYTES_PER_PROBE) / wlk / 1e9)
    return r


# --------------------------------------------------------------------------- node2vec on R-MAT 22
N_SCALE, N_LEN, N_BATCH = 22, 40, 1_000_000
N_CPU_WALKS = 131072
N_SEED = 1234 + 3
N2V_BYTES_PER_TRIAL, N2V_BYTES_PER_PROBE = 32, 8  # algorithmic bytes: one alias draw; one adjacency lookup


def make_node2vec_workload(steps_total: int, w_hi: int = (1 << 24) - 1):
    """R-MAT scale 22 (edge factor 16), Zipf(s = 1.2) weights on [1, w_hi];
    per step one update batch of 1M edges (500K absent-pair inserts + 500K
    uniform live-edge deletes) then one node2vec walk per vertex."""
    from bingo_b200 import gen
    n = 1 << N_SCALE
    src, dst = gen.rmat(N_SCALE, EDGE_FACTOR, seed=N_SEED)
    w = gen.weights(len(src), gen.W_ZIPF, 1, w_hi, 1.2, seed=N_SEED + 1)
    ug = gen.UpdateGen(n, src, dst, seed=N_SEED + 2)
    batches = [(ug.inserts(N_BATCH // 2, gen.W_ZIPF, 1, w_hi, 1.2), ug.deletes(N_BATCH // 2))
               for _ in range(steps_total)]
    return n, src, dst, w, batches


def run_node2vec(args):
    """node2vec in the plain per-job form: node2vec (p = 0.5, q = 2) walks of
    length 40 from every vertex of an R-MAT scale 22 graph with Zipf weights,
    after each 1M-edge update batch; device-timed, inputs in HBM."""
    from bingo_b200 import NODE2VEC
    world, rank, local = dist_setup()
    if rank != 0:
        return
    total = args.warmup + args.steps
    n, src, dst, w, batches = make_node2vec_workload(total)
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t_busy0 = time.time()
    r = measure_engine(args, n, src, dst, w, batches, local, app=NODE2VEC, length=N_LEN, p=0.5, q=2.0)
    clk = clocks.stop(t_busy0, time.time())
    peak, peak_src = peak_hbm()
    cpu = None
    if not args.no_cpu:
        walks = min(args.cpu_walks, N_CPU_WALKS)  # node2vec runs the plain oracle walk: a smaller sample
        c = CpuRun(n, src, dst, w).step(batches[0], walks, seed=7, app=NODE2VEC, length=N_LEN, p=0.5, q=2.0)
        cpu = {"value": c["value"], "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"one full 500K+500K update batch + {walks} node2vec walks x {N_LEN} on the CPU oracle "
                         f"(OpenMP), walk time scaled to {n} walks",
               "walk_steps_per_s": c["walk_steps_per_s"], "edge_updates_per_s": c["edge_updates_per_s"]}
    line = {"metric": "walk_steps_per_s", "value": r["value"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (r["walk_kernel_ms_per_step"] + r["update_ms_per_step"]),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {"workload": f"plain-node2vec-rmat{N_SCALE}", "scale": N_SCALE, "edge_factor": EDGE_FACTOR,
                       "m": int(len(src)), "weights": "zipf(1.2)[1,2^24)", "walks": n, "walk_len": N_LEN, "p": 0.5,
                       "q": 2.0, "batch": {"insert": N_BATCH // 2, "delete": N_BATCH // 2},
                       "form": "plain (one launch per job)"},
            "walk_steps_per_s": r["walk_steps_per_s"], "edge_updates_per_s": r["edge_updates_per_s"],
            "node2vec": {k: r[k] for k in ("trials_per_step", "probes_per_step")},
            "roofline": {"bound": "hbm", "achieved": r["algorithmic_gbs"], "peak": peak, "unit": "GB/s",
                         "frac": r["algorithmic_gbs"] / peak, "traffic": None, "peak_source": peak_src,
                         "kernel": "k_walk_plain<NODE2VEC>",
                         "bytes": f"{N2V_BYTES_PER_TRIAL} B per proposal + {N2V_BYTES_PER_PROBE} B per probe"},
            "cpu_baseline": cpu, "clocks": clk, "store_check": r["store_check"]}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- the other workloads, one line
# The default run also measures the node2vec, batched and served workloads
# and the reference's own CUDA build, each in a child process of its own
# (fresh device memory, its own clock record), and reports them as keys of
# the one JSON line.
EXTRA_RUNS = {
    "node2vec_cfg3": ["bench.py", "--workload", "node2vec", "--steps", "3", "--warmup", "3", "--no-cpu"],
    "batched_cfg4": ["bench.py", "--workload", "batched", "--steps", "3", "--warmup", "3"],
    "served_cfg5": ["bench.py", "--workload", "served", "--rates", "4000,8000,16000", "--requests", "1200"],
    "reference_cuda_cfg2": ["oracle/compare_reference_cuda.py", "--workload", "plain", "--steps", "3",
                            "--warmup", "3"],
}


def run_child(argv, timeout=900):
    t0 = time.time()
    try:
        r = subprocess.run([sys.executable] + argv, capture_output=True, text=True, timeout=timeout, cwd=ROOT)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout} s"}
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    if r.returncode or not lines:
        return {"error": f"exit {r.returncode}", "stderr_tail": r.stderr[-800:]}
    d = json.loads(lines[-1])
    d["wall_s"] = round(time.time() - t0, 1)
    return d


def summarize_extra(key, d):
    """The figures of a child run's line that the headline line carries."""
    if "error" in d or "unavailable" in d:
        return d
    keep = {"node2vec_cfg3": ("value", "unit", "ms_per_step", "walk_steps_per_s", "edge_updates_per_s", "node2vec",
                              "roofline", "config", "clocks", "store_check", "wall_s"),
            "batched_cfg4": ("value", "unit", "ms_per_step", "config", "plain", "batched", "batched_default_knobs",
                             "batched_over_plain", "clocks", "wall_s"),
            "served_cfg5": ("value", "unit", "config", "clocks", "wall_s"),
            "reference_cuda_cfg2": ("config", "reference", "ours_same_input", "clocks", "wall_s")}[key]
    out = {k: d[k] for k in keep if k in d}
    if key == "batched_cfg4" and "autotune" in d:
        out["autotune_knobs"] = {k: v for k, v in d["autotune"].items() if k != "trials"}
    if key == "served_cfg5":
        out["sweep"] = []
        for r in d["sweep"]:
            row = {k: r[k] for k in ("rate_req_s", "requests", "walk_queries", "update_batches", "update_edges")}
            for form in ("served", "plain"):
                row[form] = {k: r[form][k] for k in ("walk_p50_ms", "walk_p99_ms", "update_p50_ms", "update_p99_ms",
                                                     "walk_steps_per_s", "requests_per_s", "span_s")}
            row["served_over_plain_req_s"] = r["served"]["requests_per_s"] / r["plain"]["requests_per_s"]
            out["sweep"].append(row)
    if key == "reference_cuda_cfg2":
        ref, ours = d["reference"], d["ours_same_input"]
        out["ours_over_reference"] = {k: ours[k] / ref[k] for k in ("value", "walk_steps_per_s", "edge_updates_per_s")}
    return out


def run_extras():
    out = {}
    for key, argv in EXTRA_RUNS.items():
        out[key] = summarize_extra(key, run_child(argv))
    targets = {}
    b = out.get("batched_cfg4", {})
    if "batched_over_plain" in b:
        targets["batched_over_plain_cfg4"] = b["batched_over_plain"]
    sv = out.get("served_cfg5", {})
    if sv.get("sweep"):
        top = max(sv["sweep"], key=lambda r: r["rate_req_s"])
        targets["served_over_plain_req_s_cfg5"] = top["served_over_plain_req_s"]
    rc = out.get("reference_cuda_cfg2", {})
    if "ours_over_reference" in rc:
        targets["steps_over_reference_cuda_cfg2"] = rc["ours_over_reference"]["value"]
        targets["walk_kernel_over_reference_cuda_cfg2"] = rc["ours_over_reference"]["walk_steps_per_s"]
    out["targets"] = targets
    return out


def under_profiler() -> bool:
    """True inside an Nsight Compute (or other CUDA injection) run: the child
    workloads are then skipped, so a capture never follows them."""
    return bool(os.environ.get("CUDA_INJECTION64_PATH") or os.environ.get("NV_COMPUTE_PROFILER_PERFWORKS_DIR"))


# --------------------------------------------------------------------------- GPU arm
def run_e2e(args, g, n, src, dst, w, batches, seed, stream, dev, world):
    """The same steps through the C ABI with pinned host buffers: every step
    copies its update batch in and its slot ids and walk rows out."""
    import torch
    from bingo_b200 import DEEPWALK, PLAIN, WalkJob
    total = args.warmup + args.steps
    g.load_edges(src, dst, w, n)
    g.sync()

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).pin_memory()
        return t

    hbatches = [((pinned(i[0]), pinned(i[1]), pinned(i[2])), (pinned(d[0]), pinned(d[1]))) for i, d in batches]
    # Two host result buffers used in turn (a consumer reads one step's rows
    # while the next step runs); the engine copies each step's rows out while
    # the next step's kernels run, and bingo_sync waits for the copies.
    hout = [torch.empty((n, WALK_LEN), dtype=torch.int32).pin_memory() for _ in range(2)]
    hslots = torch.empty(BATCH_INS, dtype=torch.int32).pin_memory()

    def e2e_step(i):
        (a, b, c), (du, ds) = hbatches[i]
        g.insert_batch(a, b, c, out_slots=hslots)
        g.delete_batch(du, ds)
        g.walk_jobs([WalkJob(app=DEEPWALK, length=WALK_LEN, starts=None, n_starts=n, first=0, job_id=i, seed=seed,
                             out=hout[i % 2])], mode=PLAIN)

    for i in range(args.warmup):
        e2e_step(i)
    g.sync()
    torch.cuda.synchronize(dev)
    st2 = g.stats()
    barrier(world)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.warmup, total):
        e2e_step(i)
    g.sync()  # every result copy has landed in host memory
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    g.sync()
    st3 = g.stats()
    e2e_ms = reduce_max(e0.elapsed_time(e1), world, dev)
    e2e_steps = reduce_sum(st3["walk_steps"] - st2["walk_steps"], world, dev)
    h2d = BATCH_INS * 12 + BATCH_DEL * 8
    d2h = n * WALK_LEN * 4 + BATCH_INS * 4

    return {"value": e2e_steps / (e2e_ms / 1e3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h}


def run_ours(args):
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    from bingo_b200 import DEEPWALK, PLAIN, Graph, WalkJob

    total = args.warmup + args.steps
    n, src, dst, w, batches = make_workload(total)
    # A dedicated (non-default) stream shared by torch's events and the engine.
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    # DeepWalk only: no node2vec adjacency index, as the reference builds it
    # only for node2vec runs (NODE2VEC = 0 unless the app is node2vec,
    # include/api.h:26, src/apps.cu:14-15).
    g = Graph(device=local, synchronous=False, node2vec=False)
    g.set_stream(stream.cuda_stream)
    g.load_edges(src, dst, w, n)
    g.sync()

    def dev_i32(a):
        return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).to(dev)

    dbatches = [((dev_i32(i[0]), dev_i32(i[1]), dev_i32(i[2])), (dev_i32(d[0]), dev_i32(d[1]))) for i, d in batches]
    out = torch.empty((n, WALK_LEN), dtype=torch.int32, device=dev)
    slots = torch.empty(BATCH_INS, dtype=torch.int32, device=dev)
    seed = 0xB1460 + rank

    ev = {k: [torch.cuda.Event(enable_timing=True) for _ in range(total)] for k in ("u0", "u1", "w1")}

    def step(i):
        (a, b, c), (du, ds) = dbatches[i]
        ev["u0"][i].record(stream)
        g.insert_batch(a, b, c, out_slots=slots)
        g.delete_batch(du, ds)
        ev["u1"][i].record(stream)
        g.walk_jobs([WalkJob(app=DEEPWALK, length=WALK_LEN, starts=None, n_starts=n, first=0, job_id=i, seed=seed,
                             out=out)], mode=PLAIN)
        ev["w1"][i].record(stream)

    clocks = Clocks(local)
    clocks.start()  # samples from the warm-up to the end of the e2e timed region
    time.sleep(0.5)
    t_busy0 = time.time()
    for i in range(args.warmup):
        step(i)
    g.sync()
    torch.cuda.synchronize(dev)
    st0 = g.stats()
    barrier(world)
    torch.cuda.synchronize(dev)
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(args.warmup, total):
        step(i)
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    barrier(world)
    g.sync()
    st1 = g.stats()
    ms = t_start.elapsed_time(t_end)
    walk_ms = sum(ev["u1"][i].elapsed_time(ev["w1"][i]) for i in range(args.warmup, total))
    upd_ms = sum(ev["u0"][i].elapsed_time(ev["u1"][i]) for i in range(args.warmup, total))
    steps_local = st1["walk_steps"] - st0["walk_steps"]
    launches = st1["kernel_launches"] - st0["kernel_launches"]
    ms_max = reduce_max(ms, world, dev)
    steps_all = reduce_sum(steps_local, world, dev)
    value = steps_all / (ms_max / 1e3)

    # ---- e2e: same work through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, g, n, src, dst, w, batches, seed, stream, dev, world)
    clk = clocks.stop(t_busy0, time.time())

    # ---- the store the timed updates left behind: every invariant holds
    # (bingo_check, outside every timed region); a failing store voids the run
    t_chk = time.perf_counter()
    chk = g.check(raise_on_corrupt=False)
    store_check = {"bad_vertices": chk["bad_vertices"], "kinds": chk["kind_names"],
                   "live_edges": chk["live_edges"], "ms": (time.perf_counter() - t_chk) * 1e3}
    if chk["bad_vertices"]:
        raise SystemExit(f"bench: the graph store fails its check after the timed updates: {store_check}")

    # ---- roofline of the walk kernel
    peak, peak_src = peak_hbm()
    achieved = steps_local * BYTES_PER_STEP / (walk_ms / 1e3) / 1e9
    tps = WALK_DRAM_BYTES_PER_STEP
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": tps * steps_local / args.steps, "traffic_source": WALK_DRAM_SOURCE, "peak_source": peak_src,
            "kernel": "k_walk_plain<DEEPWALK>", "bytes_per_step": BYTES_PER_STEP}
    if tps:
        # DRAM bytes the kernel actually moves per second (ncu bytes per step x
        # live steps per second): a random 32-byte gather moves a whole sector
        # for a 4-16 byte field, so this, not the algorithmic rate, meets the
        # DRAM limit.
        roof["dram_gbs"] = tps * steps_local / (walk_ms / 1e3) / 1e9
        roof["dram_frac"] = roof["dram_gbs"] / peak

    if not args.no_gather_ceiling and world == 1:
        pr = g.probe_gather(4 << 30)
        pr["independent_gbs"] = pr["independent_sectors_per_s"] * 32 / 1e9
        pr["chain_gbs"] = pr["chain_sectors_per_s"] * 32 / 1e9
        roof["random_sector_ceiling"] = pr
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        r = CpuRun(n, src, dst, w).step(batches[0], min(args.cpu_walks, n), seed=7)
        cpu = {"value": r["value"], "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"one full 50K+50K update batch + {min(args.cpu_walks, n)} walks x {WALK_LEN} on the CPU "
                         f"oracle ({CPU_WALK_FORM})" + scaled_note(args.cpu_walks, n),
               "walk_steps_per_s": r["walk_steps_per_s"], "edge_updates_per_s": r["edge_updates_per_s"]}

    g.close()
    extras = None
    if rank == 0 and world == 1 and not args.no_extras and not under_profiler():
        extras = run_extras()

    if rank == 0:
        line = {
            "metric": "walk_steps_per_s", "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": headline_config(len(src), world),
            "walk_steps_per_s": steps_local / (walk_ms / 1e3),
            "edge_updates_per_s": (BATCH_INS + BATCH_DEL) * args.steps / (upd_ms / 1e3),
            "e2e": e2e,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": int(launches) * world,
            "store_check": store_check,
        }
        if extras is not None:
            line["other_workloads"] = extras
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "served", "node2vec"],
                    help="plain: DeepWalk on R-MAT 20 with 50K+50K update batches (default); node2vec: node2vec on "
                         "R-MAT 22 with 1M-edge batches; batched: 256 mixed jobs on R-MAT 22, batched vs plain; "
                         "served: Poisson requests on R-MAT 24, served vs plain")
    ap.add_argument("--served-scale", type=int, default=24)
    ap.add_argument("--scale", type=int, default=22,
                    help="node2vec / batched: R-MAT scale (22 = the configs; smaller for profiler captures)")
    ap.add_argument("--rates", default="500,2000,8000", help="served: request rates (req/s) to sweep")
    ap.add_argument("--requests", type=int, default=400, help="served: requests per rate")
    ap.add_argument("--p-update", type=float, default=0.05, help="served: fraction of update requests")
    ap.add_argument("--serve-budget", type=int, default=4096, help="served: output budget in MiB")
    ap.add_argument("--cpu-walks", type=int, default=1 << 20)
    ap.add_argument("--ref-walks", type=int, default=1 << 20)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-oracle baseline leg")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg (profiling runs)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the node2vec / batched / served / reference-CUDA child runs of the default workload")
    ap.add_argument("--no-gather-ceiling", action="store_true",
                    help="skip measuring the GPU's random 32-byte-sector read ceiling (4 GiB table, ~1 s)")
    args = ap.parse_args()
    global N_SCALE, B_SCALE
    N_SCALE = B_SCALE = args.scale
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.workload == "batched" and args.impl == "ours":
        run_batched(args)
    elif args.workload == "served" and args.impl == "ours":
        run_served(args)
    elif args.workload == "node2vec" and args.impl == "ours":
        run_node2vec(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
