"""The reference arm of bench.py runs on CPU (the oracle restatement, all host
threads, a bounded row sample per step) and prints the contract's JSON line;
a non-zero rank under torchrun does no work and exits 0."""
import json
import os
import subprocess
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ARGS = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
        "--workload", "water192_cut6"]


def test_reference_arm_line():
    out = subprocess.run(ARGS, capture_output=True, text=True, timeout=600, cwd=REPO)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["config"]["workload"] == "water192_cut6"
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]


def test_reference_arm_other_ranks_idle():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run(ARGS, capture_output=True, text=True, timeout=600, cwd=REPO, env=env)
    assert out.returncode == 0 and out.stdout.strip() == ""


def test_committed_traffic_summaries():
    """The DRAM-traffic summaries the bench line reads (small-case ncu
    captures scaled per workload) are consistent: the headline workload is
    present, and each scaled figure is the capture's per-unit bytes times the
    workload's units."""
    sys.path.insert(0, REPO)
    import bench
    for kernel, unit in (("k_stacked", "bytes_per_product"), ("k_tc_tiles", "bytes_per_tensor_op")):
        with open(os.path.join(REPO, "profiles", f"{kernel}_traffic.json")) as f:
            d = json.load(f)
        per = d["per_multiply_bytes"]
        assert per["water6144_cut8"] > 0 and d[unit] > 0
        assert bench.committed_traffic(kernel, "water6144_cut8") == per["water6144_cut8"]
        assert bench.committed_traffic(kernel, "no_such_workload") is None
        cap = d["capture"]
        units = cap.get("n_products", cap.get("tensor_ops"))
        total = cap.get("bytes", cap.get("read_bytes_per_multiply", 0) + cap.get("write_bytes_per_multiply", 0))
        assert abs(total / units - d[unit]) <= 1e-9 * d[unit]
