"""bench.py's JSON contract where it can run without a GPU: the reference arm (the CPU port of
the reference algorithm) and the helpers the roofline uses."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_line():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0",
                          "--ref-sample", "8"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["config"]["workload"] == "refs-ring12-water4096"


def test_roofline_helpers():
    sys.path.insert(0, ROOT)
    import bench
    from ermod_openacc_b200 import systems as S
    assert bench.profile_table("no_such_table.txt") == {}
    assert bench.bound_from_counters({}) == "unmeasured"
    assert bench.bound_from_counters({"tensor_pipe": 0.7}) == "tensor"
    assert bench.bound_from_counters({"issue_active": 0.65, "fma_pipe": 0.44}) == "sm-issue"
    assert bench.bound_from_counters({"issue_active": 0.3, "dram_frac": 0.1}) == "latency"
    assert bench.bound_from_counters({"issue_active": 0.36, "stall_mio": 4.4}) == "mio-queue"
    assert bench.bound_from_counters({"issue_active": 0.44, "l1_frac": 0.72, "stall_mio": 2.0}) == "l1-smem"
    table = bench.profile_table("kernel_counters.txt")
    assert set(table) >= {"k_pme_plane", "k_pme_lines", "k_gather_rec", "k_ecorr_tma"}
    assert "fma_pipe" not in table["k_mlp_fwd_tc"]                   # '-': not captured
    w = S.make_workload(2)
    assert 1000.0 < bench.path_bytes_per_unit(w, 12288, 4096, 1396, 2000, 12) < 1100.0
    for stage in ("gather", "bin", "pme_plane", "site_tables"):
        assert bench.kernel_bytes(stage, w, 32, 12288, 4096, 1396, 2000, 12) > 0
