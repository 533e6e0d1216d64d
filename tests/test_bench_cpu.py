"""bench.py's host-side legs, which need no GPU: the reference arm's JSON line (the binary64 oracle
port on the host cores), the error report that the precision studies attach to every CUDA mode,
and the report of the reference's own GPU algorithm (the RK4 comparator) on the oracle sample."""

import json
import subprocess
import sys
from pathlib import Path

import numpy as np

import bench
import gravlume_b200 as G
import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    run = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "1", "--cpu-sample", "64"], capture_output=True, text=True, timeout=300,
                         cwd=str(ROOT))
    assert run.returncode == 0, run.stderr[-2000:]
    line = json.loads(run.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 1
    assert line["config"]["workload"] == "kerr-newman-frame-3840x2160"
    assert set(line["cpu_baseline"]) >= {"value", "unit", "cores", "kind", "sample"}
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def oracle_as_results(ref):
    """The oracle's rows in the decoded-results layout that error_report reads."""
    F = O.F
    d = {"termination": np.nan_to_num(ref[:, F["termination"]]).astype(int),
         "escape_theta": np.arccos(np.clip(ref[:, F["escape_dz"]], -1, 1)),
         "escape_phi": np.arctan2(ref[:, F["escape_dy"]], ref[:, F["escape_dx"]]),
         "event_residual": ref[:, F["event_residual"]]}
    for k in ("frequency_ratio", "source_radius", "travel_time", "max_null_residual", "max_lz_drift",
              "max_carter_drift"):
        d[k] = ref[:, F[k]]
    return d


def test_error_report_of_the_oracle_against_itself_is_zero():
    ref, idx, _ = bench.cpu_oracle_sample(G, 96, O.hardware_threads())
    # error_report indexes the decoded results by pixel; here the 96 sampled rows stand in for them
    rows = np.full((bench.WIDTH * bench.HEIGHT, ref.shape[1]), np.nan)
    rows[idx] = ref
    rep = bench.error_report(G, oracle_as_results(rows), ref, idx)
    assert rep["rays"] == 96 and rep["class_mismatch"] == 0
    assert rep["escape_direction_rad"] < 1e-7
    for k in ("g_rel", "hit_radius", "travel_time", "max_null_residual", "max_lz_drift", "max_carter_drift"):
        assert rep[k] == 0.0, k


def test_reference_gpu_algorithm_report_on_the_oracle_sample():
    ref, idx, _ = bench.cpu_oracle_sample(G, 96, O.hardware_threads())
    rep = bench.reference_gpu_algorithm_report(G, ref, idx, O.hardware_threads())
    assert rep["rays"] == 96 and rep["class_mismatch"] == 0
    assert rep["uncertain"] == 0 and rep["step_exhaustion"] == 0
    # binary32 fixed-policy RK4: within the reference's own GPU gate on escape directions
    assert rep["escape_direction_rad"] <= 3.82e-4
    assert 50 < rep["steps_mean"] < 2048
    json.dumps(rep)
