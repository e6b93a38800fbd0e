"""Host logic of bench.py that needs no GPU: the default line's summary of
the node2vec / batched / served / reference-CUDA child runs, the profiler
guard that keeps child runs out of an ncu capture, and the reference arm's
other ranks under torchrun."""
import bench


def _served_row(rate, served_rps, plain_rps):
    form = lambda rps: {"walk_p50_ms": 1.0, "walk_p99_ms": 2.0, "update_p50_ms": 3.0, "update_p99_ms": 4.0,  # noqa
                        "walk_steps_per_s": 1e9, "requests_per_s": rps, "span_s": 0.1, "scheduler": {"x": 1},
                        "slowest_requests": [1, 2]}
    return {"rate_req_s": rate, "requests": 400, "walk_queries": 380, "update_batches": 20, "update_edges": 10,
            "served": form(served_rps), "plain": form(plain_rps)}


def test_summaries_and_targets(monkeypatch):
    lines = {
        "node2vec_cfg3": {"value": 6e9, "unit": "steps/s", "ms_per_step": 30.0, "walk_steps_per_s": 7e9,
                          "edge_updates_per_s": 5e8, "node2vec": {}, "roofline": {}, "config": {}, "clocks": {},
                          "store_check": {}, "cpu_baseline": None},
        "batched_cfg4": {"value": 7e9, "unit": "steps/s", "ms_per_step": 140.0, "config": {}, "plain": {},
                         "batched": {}, "batched_default_knobs": {}, "batched_over_plain": 2.1,
                         "autotune": {"walk_chunk": 16, "trials": [1, 2, 3]}, "clocks": {}},
        "served_cfg5": {"value": 1e10, "unit": "steps/s", "config": {}, "clocks": {},
                        "sweep": [_served_row(4000, 4000, 3900), _served_row(16000, 11000, 4000)]},
        "reference_cuda_cfg2": {"config": {}, "clocks": {},
                                "reference": {"value": 1e9, "walk_steps_per_s": 4e9, "edge_updates_per_s": 7e6},
                                "ours_same_input": {"value": 1.8e10, "walk_steps_per_s": 2.4e10,
                                                    "edge_updates_per_s": 2.5e8}},
    }
    monkeypatch.setattr(bench, "run_child", lambda argv, timeout=900: dict(
        lines[next(k for k, a in bench.EXTRA_RUNS.items() if a == argv)], wall_s=1.0))
    out = bench.run_extras()
    t = out["targets"]
    assert t["batched_over_plain_cfg4"] == 2.1
    assert abs(t["served_over_plain_req_s_cfg5"] - 11000 / 4000) < 1e-12
    assert t["steps_over_reference_cuda_cfg2"] == 18.0
    assert t["walk_kernel_over_reference_cuda_cfg2"] == 6.0
    assert "trials" not in out["batched_cfg4"]["autotune_knobs"]
    row = out["served_cfg5"]["sweep"][1]
    assert "scheduler" not in row["served"] and "slowest_requests" not in row["plain"]
    assert "cpu_baseline" not in out["node2vec_cfg3"]


def test_failed_child_is_reported_not_raised(monkeypatch):
    monkeypatch.setattr(bench, "run_child", lambda argv, timeout=900: {"error": "exit 1", "stderr_tail": "boom"})
    out = bench.run_extras()
    assert out["batched_cfg4"]["error"] == "exit 1"
    assert out["targets"] == {}


def test_profiler_guard(monkeypatch):
    monkeypatch.delenv("CUDA_INJECTION64_PATH", raising=False)
    monkeypatch.delenv("NV_COMPUTE_PROFILER_PERFWORKS_DIR", raising=False)
    assert not bench.under_profiler()
    monkeypatch.setenv("CUDA_INJECTION64_PATH", "/x/libinjection.so")
    assert bench.under_profiler()


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun with N > 1 the reference arm runs on rank 0 alone; every
    other rank exits 0 at once, prints nothing and joins no collective."""
    import os
    import subprocess
    import sys
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1", MASTER_PORT="1")
    r = subprocess.run([sys.executable, bench.__file__, "--impl", "reference", "--gpus", "2", "--steps", "2",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-800:]
    assert r.stdout.strip() == ""
