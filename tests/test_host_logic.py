"""The device tracer's per-ray state machine, compiled for the host by the test harness
(tests/native/host_trace.cpp), against the binary64 oracle: event arming and localization,
turning points, equatorial crossings, winding and drifts in all three precision modes. The same
budgets hold for the CUDA kernels in tests/test_gpu_parity.py."""

import numpy as np
import pytest

import gravlume_b200 as G
import host_harness as H
import oracle as O
from gpu_common import F, compare, config1_observation, oracle_for

BUDGETS = {
    G.Precision.FP64: dict(escape_direction_rad=1e-7, travel_time=1e-6, max_null_residual=1e-9,
                           max_lz_drift=1e-8, max_carter_drift=1e-8),
    G.Precision.MIXED: dict(escape_direction_rad=1e-6, travel_time=1e-3, max_null_residual=1e-5,
                            max_lz_drift=1e-4, max_carter_drift=1e-4),
    G.Precision.FP32: dict(escape_direction_rad=2e-3, travel_time=5e-2),
}


@pytest.fixture(scope="module")
def config1_rays():
    obs = config1_observation()
    osc, ev, sc = oracle_for(obs)
    rng = np.random.default_rng(11)
    px, py = rng.integers(0, 256, 64), rng.integers(0, 256, 64)
    states, _, _, status = O.initial_rays(osc, px, py)
    assert (status == 0).all()
    ref = O.trace_states(1.0, 0.9, 0.3, 1, O.custom_policy(1e-10, 1e-12), ev, states, -1.0,
                         threads=O.hardware_threads())
    return sc, states, ref


@pytest.mark.parametrize("precision", [G.Precision.FP64, G.Precision.MIXED, G.Precision.FP32])
def test_kernel_logic_matches_the_oracle(config1_rays, precision):
    sc, states, ref = config1_rays
    d = H.trace_states(sc, G.ReferencePolicy.frame(precision), states, -1.0)
    rep = compare(d, np.arange(len(states)), ref)
    assert rep["class_mismatch"] == 0, rep
    assert rep["radial_turnings_mismatch"] == 0 and rep["equatorial_crossings_mismatch"] == 0, rep
    for k, tol in BUDGETS[precision].items():
        assert rep[k] <= tol, (k, rep)


def test_mixed_errors_are_below_plain_fp32(config1_rays):
    sc, states, ref = config1_rays
    m = compare(H.trace_states(sc, G.ReferencePolicy.frame(G.Precision.MIXED), states, -1.0), np.arange(64), ref)
    f = compare(H.trace_states(sc, G.ReferencePolicy.frame(G.Precision.FP32), states, -1.0), np.arange(64), ref)
    # Observables set by the step-size controller (rtol 1e-6 truncation error in both modes) agree
    # within the scatter of a 64-ray maximum; the event residual, set by the localization
    # precision, is binary64-small in MIXED.
    for k in ("escape_direction_rad", "travel_time", "max_null_residual", "max_lz_drift", "max_carter_drift"):
        assert m[k] <= 1.5 * f[k], (k, m[k], f[k])
    assert m["event_residual_gpu_max"] <= 1e-3 * f["event_residual_gpu_max"]


def test_split_mixed_matches_the_oracle(config1_rays):
    """MIXED as two kernels (binary32 bulk stepping, hand-off record, binary64 completion): the
    same classes, turning points and crossings as the oracle, the one-kernel MIXED budgets, and a
    binary64 event residual."""
    sc, states, ref = config1_rays
    d = H.trace_split(sc, G.ReferencePolicy.frame(G.Precision.MIXED), states, -1.0)
    rep = compare(d, np.arange(len(states)), ref)
    assert rep["class_mismatch"] == 0, rep
    assert rep["radial_turnings_mismatch"] == 0 and rep["equatorial_crossings_mismatch"] == 0, rep
    for k, tol in BUDGETS[G.Precision.MIXED].items():
        assert rep[k] <= tol, (k, rep)
    assert rep["event_residual_gpu_max"] <= 1e-9, rep
    # every ray was finished by the binary64 completion (at least the re-taken terminal step)
    assert (d["f64_steps"] >= 1).all()


def test_split_mixed_pericentre_radius_matches_the_oracle(config1_rays):
    """The binary32 bulk stepping takes a pericentre's radius as the largest root of the radial
    potential of the step's constants of motion (Newton in binary32, with the dense-output root as
    the fallback): on the host-compiled kernel logic it has a pericentre exactly where the oracle
    has one, within 1e-5 of the oracle's radius."""
    sc, states, ref = config1_rays
    d = H.trace_split(sc, G.ReferencePolicy.frame(G.Precision.MIXED), states, -1.0)
    has = ref[:, O.F["has_turning_radius"]] == 1
    assert np.array_equal(np.isfinite(d["turning_radius"]), has)
    assert has.sum() >= 10
    otr = ref[has, O.F["turning_radius"]]
    rel = np.abs(d["turning_radius"][has] - otr) / otr
    assert rel.max() <= 1e-5, float(rel.max())


def test_split_mixed_equals_one_kernel_mixed_before_the_hand_off(config1_rays):
    """Both MIXED forms step the same binary32 pair state, so they agree to a few binary32 ulps of
    the rtol 1e-6 truncation error on every observable and take the same number of accepted steps
    within the re-taken terminal step."""
    sc, states, ref = config1_rays
    pol = G.ReferencePolicy.frame(G.Precision.MIXED)
    a = H.trace_split(sc, pol, states, -1.0)
    b = H.trace_states(sc, pol, states, -1.0)
    assert (a["termination"] == b["termination"]).all()
    assert np.all(np.abs(a["accepted_steps"] - b["accepted_steps"]) <= 2)
    assert np.nanmax(np.abs(a["travel_time"] - b["travel_time"])) < 1e-3


def test_escape_is_never_lost_across_precisions():
    """A ray leaving the escape sphere must terminate there in every mode (no step exhaustion)."""
    obs = config1_observation(width=64, height=64)
    osc, ev, sc = oracle_for(obs)
    px, py = np.meshgrid(np.arange(0, 64, 4), np.arange(0, 64, 4))
    states, _, _, _ = O.initial_rays(osc, px.ravel(), py.ravel())
    for prec in G.Precision:
        d = H.trace_states(sc, G.ReferencePolicy.frame(prec), states, -1.0)
        assert (d["termination"] != G.Termination.STEP_EXHAUSTION).all()
        esc = d["termination"] == G.Termination.ESCAPE
        assert esc.any()
        r = np.sqrt(d["x"] ** 2 + d["y"] ** 2 + d["z"] ** 2)
        assert np.all(np.abs(r[esc] - 1000.0) < 1e-2)


def test_geodesic_fixtures_through_the_kernel_logic(golden):
    for fid, policy in [("schwarzschild-scatter-b6-v1", G.ReferencePolicy.regular_v1()),
                        ("schwarzschild-scatter-near-critical-v1", G.ReferencePolicy.strict_v1()),
                        ("schwarzschild-capture-near-critical-v1", G.ReferencePolicy.strict_v1())]:
        fx = golden[fid]
        esc = float(fx["events"].get("escape_radius_m", 0.0))
        sc = G.Observation(spin=0.0, chart=G.KerrSchildChart.INGOING, observer_txyz=(0.0, 60.0, 0.0, 1.0),
                           escape_radius=esc).pack()
        st = [float(v) for v in fx["initial"]["position_txyz_m"]] + [float(v) for v in fx["initial"]["momentum_covariant"]]
        d = H.trace_states(sc, policy, [st], 1.0)
        exp, tol = fx["expected"], fx["tolerance"]
        want = G.Termination.ESCAPE if exp["termination"] == "escape" else G.Termination.HORIZON_CROSSING
        assert d["termination"][0] == want
        assert abs(d["azimuth_advance"][0] - float(exp["azimuth_advance_rad"])) <= float(tol["azimuth_advance_abs_rad"])
        if "turning_radius_m" in exp:
            assert abs(d["turning_radius"][0] - float(exp["turning_radius_m"])) <= float(tol["turning_radius_abs_m"])
        else:
            assert np.isnan(d["turning_radius"][0])
