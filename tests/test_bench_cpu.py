"""bench.py's contract on a machine without a GPU: the product arm fails
loudly (no CPU fallback), the reference arm's non-zero ranks exit without
work, and the pure helpers (plain-arm latencies, the line's config) behave."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, env_extra=None, timeout=120):
    env = dict(os.environ, **(env_extra or {}))
    env.pop("CUDA_VISIBLE_DEVICES", None)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=timeout)


def _have_gpu():
    from conftest import have_gpu

    return have_gpu()


@pytest.mark.skipif(_have_gpu(), reason="checks the behaviour without a device")
def test_product_arm_fails_loudly_without_a_device():
    r = _run(["--steps", "1", "--warmup", "3"])
    assert r.returncode != 0
    assert "no CUDA device" in r.stderr
    assert r.stdout.strip() == ""  # no bench line from a fallback


def test_reference_arm_other_ranks_exit_without_work():
    r = _run(["--impl", "reference", "--steps", "1", "--warmup", "3"],
             {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, timeout=60)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_plain_arm_latencies_follow_one_server_in_arrival_order():
    import bench

    lat, fin = bench.fifo_latencies([0.0, 0.5, 10.0], [2.0, 1.0, 1.0])
    # request 1 waits for request 0 (finish 2.0), request 2 finds the server idle
    assert lat == pytest.approx([2.0, 2.5, 1.0])
    assert fin == pytest.approx(11.0)
    assert bench.fifo_latencies([], []) == ([], 0.0)


def test_line_config_names_the_workload_and_the_replicas():
    import bench

    c1, c4 = bench.line_config(1), bench.line_config(4)
    assert c1["parallelism"] == "replicas x1" and c4["parallelism"] == "replicas x4"
    assert "workload" in c1 and c1["workload"] == c4["workload"]
    assert "L2 flushed" in c1["l2"]
