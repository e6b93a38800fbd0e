"""The C++ experiment driver (bingo_b200/bingo_driver, the reference's
instance() over the C ABI): runs every app and update mode on the GPU (with
the store check after every iteration on request), reads an edge-list file,
and fails with a clear status when there is no GPU."""
import json
import os
import subprocess

import numpy as np
import pytest

from bingo_b200 import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "bingo_b200", "bingo_driver")


def _run(*args, timeout=300):
    if not os.path.exists(DRIVER):  # a build output, not part of the source tree
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "bingo_b200"), DRIVER], check=True)
    return subprocess.run([DRIVER, *args], capture_output=True, text=True, timeout=timeout)


def test_driver_without_gpu_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = _run("d", "-r", "8", "-k", "1")
    assert r.returncode == 2
    assert "no CUDA device" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("app,mode,extra", [("d", "-m", []), ("n", "-i", []), ("p", "-d", []), ("s", "-m", []),
                                            ("d", "-m", ["-f"]), ("n", "-m", ["-c"])])
def test_driver_runs_the_reference_loop(app, mode, extra):
    r = _run(app, "-r", "12", mode, "-b", "4000", "-k", "3", "-l", "40", *extra)
    assert r.returncode == 0, r.stderr
    assert "Random walk in" in r.stderr and "Evaluation time" in r.stderr
    d = json.loads(r.stdout.strip().splitlines()[-1])
    per = d["batch"] * d["iterations"]
    want = d["m"] + (per if mode in ("-m", "-i") else 0) - (per if mode in ("-m", "-d") else 0)
    assert d["live_edges"] == want
    assert d["walk_steps"] > 0 and d["walk_steps_per_s"] > 0
    assert d["store_checks"] == (1 + d["iterations"] if "-c" in extra else 0)


@pytest.mark.gpu
def test_driver_reads_an_edge_list(tmp_path):
    src, dst = gen.rmat(11, 8, seed=5)
    p = tmp_path / "g.txt"
    with open(p, "w") as f:
        f.write("# a SNAP-style header\n")
        np.savetxt(f, np.stack([src, dst], 1), fmt="%d")
    r = _run("d", "-g", str(p), "-b", "1000", "-k", "2", "-o")
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    d = json.loads(lines[-1])
    assert d["m"] == len(src) and d["n"] == int(max(src.max(), dst.max())) + 1
    assert len(lines) == 11  # ten printed walks, then the summary
