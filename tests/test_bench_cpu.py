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
    ref, idx, _ = bench.cpu_oracle_sample(96, O.hardware_threads())
    # error_report indexes the decoded results by pixel; here the 96 sampled rows stand in for them
    rows = np.full((bench.WIDTH * bench.HEIGHT, ref.shape[1]), np.nan)
    rows[idx] = ref
    rep = bench.error_report(oracle_as_results(rows), ref, idx)
    assert rep["rays"] == 96 and rep["class_mismatch"] == 0
    assert rep["escape_direction_rad"] < 1e-7
    for k in ("g_rel", "hit_radius", "travel_time", "max_null_residual", "max_lz_drift", "max_carter_drift"):
        assert rep[k] == 0.0, k


def test_reference_gpu_algorithm_report_on_the_oracle_sample():
    ref, idx, _ = bench.cpu_oracle_sample(96, O.hardware_threads())
    rep = bench.reference_gpu_algorithm_report(ref, idx, O.hardware_threads())
    assert rep["rays"] == 96 and rep["class_mismatch"] == 0
    assert rep["uncertain"] == 0 and rep["step_exhaustion"] == 0
    # binary32 fixed-policy RK4: within the reference's own GPU gate on escape directions
    assert rep["escape_direction_rad"] <= 3.82e-4
    assert 50 < rep["steps_mean"] < 2048
    json.dumps(rep)


def test_reference_arm_maps_no_product_library():
    """The reference arm runs the oracle alone: neither the package nor libglc.so is loaded."""
    script = ("import runpy, sys\n"
              "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', '--cpu-sample', '32']\n"
              "runpy.run_path('bench.py', run_name='__main__')\n"
              "maps = open('/proc/self/maps').read()\n"
              "print('GLC_MAPPED', 'libglc' in maps, 'gravlume_b200' in sys.modules, 'libgravlume_oracle' in maps)\n")
    run = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert run.returncode == 0, run.stderr[-2000:]
    last = run.stdout.strip().splitlines()[-1]
    assert last == "GLC_MAPPED False False True", last


def test_oracle_job_places_the_observer_like_the_product_scene():
    """The reference arm's oracle-only scene equals the one built from the product's Observation."""
    osc, ev = bench.oracle_job()
    obs = bench.make_observation(G)
    assert list(osc.observer_txyz) == [float(v) for v in obs.observer_txyz]
    assert osc.vertical_fov == obs.vertical_fov
    assert ev.surface_inner == obs.surface.inner_radius


def test_headline_line_is_short():
    """The last stdout line of the GPU arm stays well under the 1500 characters a log tail keeps,
    with full-length floats in every field."""
    x = 1.0 / 3.0
    roof = {"bound": "fp32_fma", "achieved": x, "peak": x, "unit": "TFLOP/s", "frac": x, "traffic": x * 1e9,
            "hbm_view": {"frac": x}}
    clk = {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 1000}
    e2e = {"value": x, "unit": "Mrays/s", "h2d_bytes_per_step": 123456, "d2h_bytes_per_step": 1658880000}
    policy = {"position_rtol": 1e-6, "persistent": 0}
    line = bench.make_headline(x * 100, 1, 20, 5, x * 10, "mixed", policy, 60, clk, e2e, roof)
    line["cpu_baseline"] = bench.rounded({"value": x, "unit": "Mrays/s", "cores": 16, "kind": "port",
                                          "sample": "2048 seeded pixels, rtol 1e-10"})
    text = json.dumps(line)
    assert len(text) < 1024, len(text)
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "gpu_launches", "clocks", "e2e", "roofline",
                "cpu_baseline"):
        assert key in line, key
    assert set(line["roofline"]) >= {"bound", "achieved", "peak", "unit", "frac", "traffic"}
