"""The reference's own CUDA build next to this engine on identical input.

TEST INFRASTRUCTURE: runs oracle/_ref/ref_harness (the reference's headers
compiled by `make -C oracle ref`, see ref_harness.cu) as a measured
baseline, then this engine through bench.py's measure_engine on the same
graph and batches. The product never runs anything here.

    python oracle/compare_reference_cuda.py [--workload plain|node2vec|small] [--steps K] [--warmup W]

plain: DeepWalk on R-MAT 20 with weights log-uniform in [1, 2^16) (the
reference's MAXLOG = 16) and 50K + 50K update batches; node2vec: R-MAT 22,
Zipf weights below 2^16, 1M-edge batches, walk length 80 (the reference's
compile-time LEN); small: DeepWalk on R-MAT 14 (16,384 vertices, edge factor
16) with weights uniform in [1, 1024] and 10K + 10K update batches, one walk
of length 80 per vertex (its whole state fits in L2, so this measures launch
and L2-resident work, not HBM). Prints one JSON line.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from bench import (BATCH_DEL, BATCH_INS, EDGE_FACTOR, N_BATCH, N_SCALE, SCALE, WALK_LEN, WORKLOAD,  # noqa: E402
                   Clocks, dist_setup, make_node2vec_workload, make_workload, measure_engine)

REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")

SMALL = dict(scale=14, ef=16, seed=1235, lo=1, hi=1024, k=10_000)


def make_small_workload(steps_total):
    """R-MAT 14, uniform [1, 1024] weights, 10K absent-pair inserts + 10K
    live-edge deletes per step (the parity tests' small DeepWalk case)."""
    from bingo_b200 import gen
    n = 1 << SMALL["scale"]
    src, dst = gen.rmat(SMALL["scale"], SMALL["ef"], seed=SMALL["seed"])
    w = gen.weights(len(src), gen.W_UNIFORM, SMALL["lo"], SMALL["hi"], seed=SMALL["seed"] + 1)
    ug = gen.UpdateGen(n, src, dst, seed=SMALL["seed"] + 2)
    batches = [(ug.inserts(SMALL["k"], gen.W_UNIFORM, SMALL["lo"], SMALL["hi"]), ug.deletes(SMALL["k"]))
               for _ in range(steps_total)]
    return n, src, dst, w, batches


def run_reference_cuda(args):
    """The reference's own CUDA build (oracle/_ref/ref_harness, compiled from
    the reference sources) on the same GPU, on this workload with weights
    capped below 2^16 (its MAXLOG = 16 bit groups), next to this engine on
    the identical input. The reference walks every vertex once per step with
    its deepwalkKernel<<<512,128>>> (timed with CUDA events) and applies each
    batch with its host insert()/deleteE() wrappers (timed on the host: they
    sort, grow vertices and synchronise on the host by design)."""
    import struct
    import tempfile
    world, rank, local = dist_setup()
    if rank != 0:
        return
    if not os.path.exists(REF_HARNESS):
        print(json.dumps({"impl": "reference-cuda", "unavailable": "oracle/_ref/ref_harness not built "
                          "(make -C oracle ref needs the reference sources)"}))
        return
    total = args.warmup + args.steps
    w_hi = 1 << 16
    n2v = args.workload == "node2vec"
    if n2v:  # node2vec on R-MAT 22 within the reference's limits: weights < 2^16 (MAXLOG), its fixed LEN = 80
        n, src, dst, w, batches = make_node2vec_workload(total, w_hi=w_hi - 1)
    elif args.workload == "small":
        n, src, dst, w, batches = make_small_workload(total)
    else:
        n, src, dst, w, batches = make_workload(total, w_hi=w_hi)
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        with open(inp, "wb") as f:
            f.write(b"BREF")
            f.write(struct.pack("<IIQfI", 1, n, len(src), 0.4, 1 if n2v else 0))
            f.write(np.stack([src, dst, w], 1).astype("<u4").tobytes())
            for i, (ins, dels) in enumerate(batches):
                f.write(struct.pack("<IQ", 1, len(ins[0])))
                f.write(np.stack(ins, 1).astype("<u4").tobytes())
                f.write(struct.pack("<IQ", 2, len(dels[0])))
                f.write(np.stack(dels, 1).astype("<u4").tobytes())
                f.write(struct.pack("<IIIQ", 4, 1 if n2v else 0, 1, 1000 + i))
            f.write(struct.pack("<I", 0))
        clocks = Clocks(local)
        clocks.start()
        time.sleep(0.3)
        t_busy0 = time.time()
        r = subprocess.run([REF_HARNESS, inp, "-"], capture_output=True, text=True, timeout=1800)
        clk_ref = clocks.stop(t_busy0, time.time())
    if r.returncode:
        print(json.dumps({"impl": "reference-cuda", "unavailable": f"ref_harness exited {r.returncode}: "
                          + r.stderr.strip().splitlines()[-1][:200] if r.stderr.strip() else "no message"}))
        return
    ops = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    ins_s = [o["wall_s"] for o in ops if o["op"] == "insert"][args.warmup:]
    del_s = [o["wall_s"] for o in ops if o["op"] == "delete"][args.warmup:]
    walks = [o for o in ops if o["op"] == "walk"][args.warmup:]
    walk_s = sum(o["kernel_ms"] for o in walks) / 1e3
    steps = sum(o["steps"] for o in walks)
    upd_per_step = sum(len(b[0][0]) + len(b[1][0]) for b in batches[args.warmup:]) / max(len(walks), 1)
    ref = {"value": steps / (walk_s + sum(ins_s) + sum(del_s)), "walk_steps_per_s": steps / walk_s,
           "edge_updates_per_s": upd_per_step * len(walks) / (sum(ins_s) + sum(del_s)),
           "walk_kernel_ms_per_step": walk_s * 1e3 / len(walks),
           "update_wall_ms_per_step": (sum(ins_s) + sum(del_s)) * 1e3 / len(walks),
           "steps_per_walk_phase": steps / len(walks)}
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    t_busy0 = time.time()
    if n2v:
        from bingo_b200 import NODE2VEC
        ours = measure_engine(args, n, src, dst, w, batches, local, app=NODE2VEC, length=WALK_LEN, p=0.5, q=2.0)
        cfg = {"workload": f"plain-node2vec-rmat{N_SCALE}-w16", "scale": N_SCALE, "edge_factor": EDGE_FACTOR,
               "weights": "zipf(1.2)[1,2^16)", "walks": n, "walk_len": WALK_LEN, "p": 0.5, "q": 2.0,
               "batch": {"insert": N_BATCH // 2, "delete": N_BATCH // 2},
               "note": "walk length 80 = the reference's compile-time LEN (include/api.h:12); its node2vec tests "
                       "prev in N(cur) with a load-time hash (include/operation.cuh:313), so its step counts "
                       "and acceptance differ from the exact node2vec here"}
    elif args.workload == "small":
        ours = measure_engine(args, n, src, dst, w, batches, local)
        cfg = {"workload": "plain-deepwalk-rmat14", "scale": SMALL["scale"], "edge_factor": SMALL["ef"],
               "weights": "uniform[1,1024]", "walks": n, "walk_len": WALK_LEN,
               "batch": {"insert": SMALL["k"], "delete": SMALL["k"]}, "l2": "whole state L2-resident"}
    else:
        ours = measure_engine(args, n, src, dst, w, batches, local)
        cfg = {"workload": WORKLOAD + "-w16", "scale": SCALE, "edge_factor": EDGE_FACTOR,
               "weights": "loguniform[1,2^16)", "walks": n, "walk_len": WALK_LEN,
               "batch": {"insert": BATCH_INS, "delete": BATCH_DEL}}
    clk_ours = clocks.stop(t_busy0, time.time())
    line = {"impl": "reference-cuda", "metric": "walk_steps_per_s", "value": ref["value"], "unit": "steps/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "config": cfg, "reference": ref, "ours_same_input": ours,
            "clocks": {"reference": clk_ref, "ours": clk_ours}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="plain", choices=["plain", "node2vec", "small"])
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    run_reference_cuda(ap.parse_args())


if __name__ == "__main__":
    main()
