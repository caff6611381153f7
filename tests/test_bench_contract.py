"""The reference arm of bench.py (the CPU restatement timed on the host
cores) prints one JSON line with the keys the benchmark contract names."""
import json
import os
import subprocess
import sys


def test_reference_arm_prints_the_contract_line():
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    # by default the arm runs the GPU arm's own workload (--n-side); a small
    # one here keeps the CPU suite fast
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--n-side", "6"],
                         cwd=root, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["same_config"] and line["config"]["n_side"] == 6
    assert line["config"]["dof"] == 6 ** 3 * 8 ** 3 * 5
    assert line["cpu_baseline"]["value"] == line["value"] and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_stage_kernel_names_and_bytes_per_node():
    """Every kernel choice the solver resolves to (1-4) has a roofline name,
    and the algorithmic bytes per node match the stated figures: 3-D N=7
    FP64 272 B (Q and carry read + written, 11 metric terms, face geometry
    spread over the nodes), 3-D N=4 FP64 286.4 B, FP32 half of those."""
    import importlib.util
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(root, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert sorted(bench.STAGE_KERNELS) == [1, 2, 3, 4]
    assert bench.bytes_per_node(3, 7, 8) == 272.0
    assert abs(bench.bytes_per_node(3, 4, 8) - 286.4) < 1e-9
    assert bench.bytes_per_node(3, 7, 4) == 136.0
