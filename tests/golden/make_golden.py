"""Generate the golden fixtures in tests/golden/ from the reference's own CUDA
build.

oracle/_ref/ref_harness is built from the reference sources where they lie
(`make -C oracle ref`, needs the reference tree) and travels with the repo to
the GPU machine. This script writes seeded inputs in the harness format, runs
the harness, and stores the reference's NodeData state after the load and
after every update batch:

    python tests/golden/make_golden.py --out <dir>      # needs a GPU

Each case becomes ref_<name>.npz (inputs + every dump). The config-1 sized
case is too large to store whole, so only SHA-256 digests of its dumps are
kept (ref_rmat14_digest.json); the test replays it on the CPU oracle.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import struct
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from bingo_b200 import gen  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")


def rmat_case(scale, ef, seed, dist, lo, hi, rounds, k_ins, k_del, rate=0.4):
    n = 1 << scale
    src, dst = gen.rmat(scale, ef, seed=seed)
    w = gen.weights(len(src), dist, lo, hi, 1.2, seed=seed + 1)
    ug = gen.UpdateGen(n, src, dst, seed=seed + 2)
    ops = []
    for _ in range(rounds):
        ops.append(("ins",) + ug.inserts(k_ins, dist, lo, hi, 1.2))
        ops.append(("del",) + ug.deletes(k_del))
    return dict(n=n, rate=rate, src=src, dst=dst, w=w, ops=ops)


def edge_case():
    """Hand-made corner cases: single edge, dense groups, a vertex empty at
    load, weights above the load-time bit length, capacity growth, deleting
    every edge of a vertex, deleting the last member of a group, duplicate
    (u, v) pairs."""
    n = 64
    E = []
    E.append((0, 9, 5))                                   # single edge
    E += [(1, 10 + i, 3) for i in range(20)]              # dense bits 0,1
    E += [(2, 30 + i, i + 1) for i in range(10)]          # mixed weights
    E += [(4, 40 + i, 1 << i) for i in range(5)]          # LOGT = 5
    E += [(5, 50 + i, 7) for i in range(3)]               # all deleted later
    E += [(6, (7 + i) % n, (i % 13) + 1) for i in range(17)]  # capacity 32 at load
    E += [(7, 8, 1), (7, 9, 2)]
    src = np.array([e[0] for e in E], np.uint32)
    dst = np.array([e[1] for e in E], np.uint32)
    w = np.array([e[2] for e in E], np.uint32)
    # slots: vertex 5 has slots 0..2, vertex 4 slots 0..4, vertex 7 slots 0..1
    ins1 = [(3, 1, 6), (3, 2, 1), (4, 60, 1023), (6, 1, 2), (7, 8, 1)] + [(6, (20 + i) % n, 5) for i in range(20)]
    del1 = [(5, 0), (5, 2), (5, 1), (4, 4), (7, 1), (0, 0)]
    ins2 = [(5, 33, 4), (0, 10, 8), (1, 2, 3), (3, 4, 2)]
    del2 = [(1, 0), (1, 19), (1, 5), (6, 17), (6, 36), (3, 0)]
    ops = []
    for kind, lst in (("ins", ins1), ("del", del1), ("ins", ins2), ("del", del2)):
        cols = list(zip(*lst))
        ops.append((kind,) + tuple(np.array(c, np.uint32) for c in cols))
    return dict(n=n, rate=0.4, src=src, dst=dst, w=w, ops=ops)


CASES = {
    "rmat10_u1024": lambda: rmat_case(10, 16, 101, gen.W_UNIFORM, 1, 1024, 3, 300, 300),
    "rmat9_u65535": lambda: rmat_case(9, 8, 202, gen.W_UNIFORM, 1, 65535, 2, 200, 200),
    "rmat8_rate01": lambda: rmat_case(8, 16, 303, gen.W_LOGUNIFORM, 1, 1 << 15, 2, 150, 150, rate=0.1),
    "edge": edge_case,
}

# The small DeepWalk workload: R-MAT scale 14, edge factor 16, uniform [1,1024],
# one batch of 10K absent-pair inserts and 10K uniform deletes.
RMAT14 = dict(scale=14, ef=16, seed=1234 + 1, lo=1, hi=1024, k=10000)


def rmat14_case():
    c = RMAT14
    return rmat_case(c["scale"], c["ef"], c["seed"], gen.W_UNIFORM, c["lo"], c["hi"], 1, c["k"], c["k"])


def write_input(path, case):
    with open(path, "wb") as f:
        f.write(b"BREF")
        f.write(struct.pack("<IIQfI", 1, case["n"], len(case["src"]), case["rate"], 0))
        f.write(np.stack([case["src"], case["dst"], case["w"]], 1).astype("<u4").tobytes())
        for op in case["ops"]:
            f.write(struct.pack("<I", 3))  # dump before the op (first: after load)
            if op[0] == "ins":
                f.write(struct.pack("<IQ", 1, len(op[1])))
                f.write(np.stack(op[1:4], 1).astype("<u4").tobytes())
            else:
                f.write(struct.pack("<IQ", 2, len(op[1])))
                f.write(np.stack(op[1:3], 1).astype("<u4").tobytes())
        f.write(struct.pack("<II", 3, 0))


def run_harness(case, work, name):
    inp = os.path.join(work, f"{name}.bin")
    out = os.path.join(work, f"{name}.dump")
    write_input(inp, case)
    r = subprocess.run([HARNESS, inp, out], capture_output=True, text=True, timeout=600)
    if r.returncode:
        raise RuntimeError(f"ref_harness failed on {name}: {r.stderr}")
    return po.read_ref_dumps(out), r.stdout


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name, make in CASES.items():
        case = make()
        dumps, log = run_harness(case, args.out, name)
        assert len(dumps) == len(case["ops"]) + 1
        arrays = dict(src=case["src"], dst=case["dst"], w=case["w"])
        kinds = []
        for i, op in enumerate(case["ops"], start=1):
            kinds.append(op[0])
            for j, col in zip("abc", op[1:]):
                arrays[f"op{i}_{j}"] = col
        for i, d in enumerate(dumps):
            for k in po.REF_DUMP_FIELDS:
                arrays[f"dump{i}_{k}"] = d[k]
        meta = dict(n=case["n"], rate=case["rate"], ops=kinds, source="oracle/_ref/ref_harness")
        np.savez_compressed(os.path.join(args.out, f"ref_{name}.npz"), meta=json.dumps(meta), **arrays)
        print(name, "ok", len(dumps), "dumps")
    case = rmat14_case()
    dumps, log = run_harness(case, args.out, "rmat14")
    rec = dict(config=RMAT14, inputs={k: digest(case[k]) for k in ("src", "dst", "w")},
               ops=[{"kind": op[0], "cols": [digest(c) for c in op[1:]]} for op in case["ops"]],
               dumps=[{k: digest(d[k]) for k in po.REF_DUMP_FIELDS} for d in dumps], harness_log=log)
    with open(os.path.join(args.out, "ref_rmat14_digest.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print("rmat14 ok")


if __name__ == "__main__":
    main()
