"""Pins the CPU oracle against the reference's golden fixtures and closed forms (no GPU).

Each test restates one of the reference's own oracle tests:
crates/gravlume-reference/tests/fixture_tests.rs, geodesic_tests.rs,
surface_observable_tests.rs, and the unit tests in geodesic.rs / surface.rs / policy.rs.
"""

import math

import numpy as np
import pytest

import oracle as O

F = O.F
EPS = np.finfo(np.float64).eps


def fixture_state(fx):
    pos = [float(v) for v in fx["initial"]["position_txyz_m"]]
    mom = [float(v) for v in fx["initial"]["momentum_covariant"]]
    return pos + mom


def fixture_events(fx):
    esc = fx["events"].get("escape_radius_m")
    return O.events(escape_radius=float(esc) if esc is not None else None)


def run_geodesic(fx, policy):
    st = fixture_state(fx)
    sp = fx["spacetime"]
    out = O.trace_states(float(sp["mass_m"]), float(sp["spin_m"]), float(sp["charge_m"]), 0,
                         policy, fixture_events(fx), [st], 1.0)
    return out[0]


def accepts(fx, row):
    """ExpectedOutcome::accepts (crates/gravlume-reference/src/fixture.rs:230-259)."""
    exp, tol = fx["expected"], fx["tolerance"]
    term = {"escape": O.ESCAPE, "horizon-crossing": O.HORIZON}[exp["termination"]]
    if row[F["termination"]] != term:
        return False
    if abs(row[F["azimuth_advance"]] - float(exp["azimuth_advance_rad"])) > float(tol["azimuth_advance_abs_rad"]):
        return False
    if "turning_radius_m" in exp:
        if not row[F["has_turning_radius"]]:
            return False
        if abs(row[F["turning_radius"]] - float(exp["turning_radius_m"])) > float(tol["turning_radius_abs_m"]):
            return False
    elif row[F["has_turning_radius"]]:
        return False
    if "event_radius_m" in exp:
        r = math.sqrt(row[F["x"]] ** 2 + row[F["y"]] ** 2 + row[F["z"]] ** 2)  # spin 0: r = |x|
        if abs(r - float(exp["event_radius_m"])) > float(tol["event_radius_abs_m"]):
            return False
    return True


def escape_angle(a, b):
    da = np.array([a[F["escape_dx"]], a[F["escape_dy"]], a[F["escape_dz"]]])
    db = np.array([b[F["escape_dx"]], b[F["escape_dy"]], b[F["escape_dz"]]])
    c = np.cross(da, db)
    return math.atan2(np.linalg.norm(c), float(np.dot(da, db)))


def comparison_issues(regular, strict):
    """ReferenceComparison::baseline_v1 budgets (crates/gravlume-reference/src/comparison.rs:66-145)."""
    issues = []
    if regular[F["termination"]] != strict[F["termination"]]:
        issues.append("termination")
    pos_r = regular[F["x"]:F["z"] + 1]
    pos_s = strict[F["x"]:F["z"] + 1]
    if np.linalg.norm(pos_r - pos_s) > 2e-9:
        issues.append("event-position")
    if regular[F["termination"]] == O.ESCAPE and escape_angle(regular, strict) > 2e-9:
        issues.append("escape-direction")
    if abs(regular[F["travel_time"]] - strict[F["travel_time"]]) > 2e-8:
        issues.append("travel-time")
    if regular[F["termination"]] == O.SURFACE:
        if abs(regular[F["source_radius"]] - strict[F["source_radius"]]) > 2e-9:
            issues.append("anchor")
        g0, g1 = regular[F["frequency_ratio"]], strict[F["frequency_ratio"]]
        if abs(g0 - g1) / g0 > 2e-9:
            issues.append("frequency-ratio")
    for k in ("max_null_residual", "max_energy_drift", "max_lz_drift", "max_carter_drift"):
        if max(regular[F[k]], strict[F[k]]) > 5e-9:
            issues.append(k)
    return issues


def default_observation_scene(fx):
    sp, ob, vp = fx["spacetime"], fx["observer"], fx["viewport"]
    return O.scene(mass=float(sp["mass_m"]), spin=float(sp["spin_m"]), charge=float(sp["charge_m"]),
                   chart=0, observer_oblate=(float(ob["oblate_radius_m"]), float(ob["polar_angle_rad"]),
                                             float(ob["azimuth_rad"])),
                   target=[float(v) for v in ob["target_txyz_m"]], width=vp["width"],
                   height=vp["height"], vertical_fov=float(vp["vertical_fov_rad"]))


def test_policy_refinement_rules_are_versioned():
    r, s = O.regular_v1(), O.strict_v1()
    assert s.position_rtol == r.position_rtol / 16 and s.momentum_atol == r.momentum_atol / 16
    assert s.maximum_step == 0.25
    assert s.maximum_accepted_steps == 2 * r.maximum_accepted_steps
    assert s.maximum_consecutive_rejects == 2 * r.maximum_consecutive_rejects
    assert s.event_affine_tolerance == r.event_affine_tolerance / 4
    assert s.event_tie_tolerance == r.event_tie_tolerance / 4
    assert r.singularity_guard == 2.0 ** -40


def test_regular_schwarzschild_fixture_and_strict_refinement_meet_the_oracle(golden):
    fx = golden["schwarzschild-scatter-b6-v1"]
    regular = run_geodesic(fx, O.regular_v1())
    assert regular[F["termination"]] == O.ESCAPE
    assert regular[F["event_bracket"]] <= O.regular_v1().event_affine_tolerance
    assert regular[F["event_residual"]] <= 5e-12
    assert int(regular[F["event_candidates"]]) == 1 << 3  # escape only: not ambiguous
    assert accepts(fx, regular)
    assert regular[F["max_null_residual"]] < 5e-9
    strict = run_geodesic(fx, O.strict_v1())
    assert comparison_issues(regular, strict) == []


def test_near_critical_pair_preserves_the_independent_discrete_classification(golden):
    esc = golden["schwarzschild-scatter-near-critical-v1"]
    cap = golden["schwarzschild-capture-near-critical-v1"]
    e = run_geodesic(esc, O.strict_v1())
    c = run_geodesic(cap, O.strict_v1())
    assert e[F["termination"]] == O.ESCAPE and accepts(esc, e)
    assert c[F["termination"]] == O.HORIZON and accepts(cap, c)
    assert c[F["has_turning_radius"]] == 0


def test_travel_time_is_independent_of_the_coordinate_time_origin(golden):
    fx = golden["schwarzschild-scatter-b6-v1"]
    st = np.array([fixture_state(fx)] * 2)
    st[1, 0] = 1.0e300
    out = O.trace_states(1.0, 0.0, 0.0, 0, O.regular_v1(), fixture_events(fx), st, 1.0)
    assert out[0, F["termination"]] == out[1, F["termination"]]
    assert out[1, F["travel_time"]] > 0
    assert abs(out[1, F["travel_time"]] - out[0, F["travel_time"]]) <= 2e-8


def test_turning_radius_is_dense_localized_for_negative_affine_traversal(golden):
    fx = golden["schwarzschild-scatter-b6-v1"]
    fwd = O.trace_states(1.0, 0, 0, 0, O.strict_v1(), fixture_events(fx), [fixture_state(fx)], 1.0)[0]
    back = O.trace_states(1.0, 0, 0, 0, O.strict_v1(), fixture_events(fx), [fwd[F["t"]:F["p_z"] + 1]], -1.0)[0]
    assert back[F["termination"]] == O.ESCAPE
    assert abs(back[F["turning_radius"]] - fwd[F["turning_radius"]]) <= 5e-11


def test_default_observation_fixture_matches_its_80_digit_values(golden):
    fx = golden["kerr-exterior-observation-v1"]
    sc = default_observation_scene(fx)
    info = O.observer_info(sc)
    tol = float(fx["tolerance"]["radius_abs_m"])
    for got, exp in zip(list(info.event)[1:], fx["expected"]["observer_cartesian_xyz_m"]):
        assert abs(got - float(exp)) <= tol
    assert abs(info.g_tt - float(fx["expected"]["observer_g_tt"])) <= tol
    assert abs(info.outer_horizon - float(fx["expected"]["outer_horizon_radius_m"])) <= tol
    assert info.gram_residual <= float(fx["tolerance"]["frame_gram_max_abs"])
    w, h = fx["viewport"]["width"], fx["viewport"]["height"]
    _, freq, res, status = O.initial_rays(sc, [w // 2], [h // 2])
    assert status[0] == 0
    assert res[0] <= float(fx["tolerance"]["initial_null_normalized_abs"])
    assert abs(freq[0] - 1.0) <= 32 * EPS


def test_observation_traces_backward_without_flipping_photon_time_orientation(golden):
    fx = golden["kerr-exterior-observation-v1"]
    sc = default_observation_scene(fx)
    ev = O.events(escape_radius=200.0)
    reg, st = O.trace_pixels(sc, O.regular_v1(), ev, [0], [0])
    strict, _ = O.trace_pixels(sc, O.strict_v1(), ev, [0], [0])
    r = reg[0]
    assert st[0] == 0
    assert r[F["termination"]] == O.ESCAPE
    assert r[F["affine_parameter"]] < 0 and r[F["travel_time"]] > 0
    d = np.array([r[F["escape_dx"]], r[F["escape_dy"]], r[F["escape_dz"]]])
    pos = np.array([r[F["x"]], r[F["y"]], r[F["z"]]])
    assert abs(float(d @ d) - 1.0) <= 8 * EPS
    assert float(pos @ d) > 0
    assert comparison_issues(r, strict[0]) == []


def test_surface_fixture_regular_and_strict_close_the_vacuum_radiance_chain(golden):
    base = golden["kerr-exterior-observation-v1"]
    fx = golden["kerr-equatorial-surface-observable-v1"]
    sc = default_observation_scene(base)
    surf = (float(fx["surface"]["inner_radius_m"]), float(fx["surface"]["outer_radius_m"]))
    ev = O.events(escape_radius=200.0, surface=surf, intensity_at_six=float(fx["emission"]["intensity_at_6m"]))
    exp, tol = fx["expected"], fx["tolerance"]
    rows = []
    for pol in (O.regular_v1(), O.strict_v1()):
        out, status = O.trace_pixels(sc, pol, ev, [fx["sample"]["x"]], [fx["sample"]["y"]])
        r = out[0]
        assert status[0] == 0 and r[F["termination"]] == O.SURFACE and r[F["surface_status"]] == 1
        assert abs(r[F["travel_time"]] - float(exp["travel_time_m"])) <= float(tol["travel_time_abs_m"])
        assert abs(r[F["source_radius"]] - float(exp["source_radius_m"])) <= float(tol["source_coordinate_abs_m"])
        daz = (r[F["source_azimuth"]] - float(exp["source_azimuth_rad"]) + math.pi) % (2 * math.pi) - math.pi
        assert abs(daz) <= float(tol["source_azimuth_abs_rad"])
        g = float(exp["frequency_ratio"])
        assert abs(r[F["frequency_ratio"]] - g) / g <= float(tol["frequency_ratio_rel"])
        assert abs(r[F["emitted_intensity"]] - float(exp["emitted_bolometric_intensity"])) <= float(tol["bolometric_intensity_abs"])
        assert abs(r[F["observed_intensity"]] - float(exp["observed_bolometric_intensity"])) <= float(tol["bolometric_intensity_abs"])
        rows.append(r)
    assert comparison_issues(rows[0], rows[1]) == []


def test_weak_field_scattering_converges_to_the_leading_four_m_over_b_deflection():
    R, b = 1000.0, 50.0
    pt = b / R
    f = 2.0 / R
    quad = f * f - (1.0 - f) * (pt * pt - 1.0 - f)
    pr = (f - math.sqrt(quad)) / (1.0 - f)
    out = O.trace_states(1.0, 0, 0, 0, O.regular_v1(), O.events(escape_radius=R),
                         [[0, R, 0, 0, -1.0, pr, pt, 0]], 1.0)[0]
    assert out[F["termination"]] == O.ESCAPE
    flat = math.pi - 2.0 * math.asin(b / R)
    deflection = out[F["azimuth_advance"]] - flat
    assert abs(deflection - 4.0 / b) <= 0.08 * 4.0 / b


def test_equatorial_surface_is_localized_as_a_distinct_terminal_event():
    out = O.trace_states(1.0, 0, 0, 0, O.regular_v1(), O.events(surface=(5.0, 60.0)),
                         [[0, 50, 0, 1, -1, -0.9, 0, -0.2]], 1.0)[0]
    assert out[F["termination"]] == O.SURFACE
    assert abs(out[F["z"]]) <= 2e-11


def test_accepted_step_limit_is_a_typed_terminal_condition():
    pol = O.regular_v1()
    pol.maximum_accepted_steps = 1
    out = O.trace_states(1.0, 0, 0, 0, pol, O.events(), [[0, 50, 0, 0, -1, -0.99, 0.1, 0]], 1.0)[0]
    assert out[F["termination"]] == O.STEP_EXHAUSTION
    assert out[F["accepted_steps"]] == 1


def test_superextremal_ring_approach_stops_at_the_singularity_guard():
    out = O.trace_states(1.0, 2.0, 0, 0, O.regular_v1(), O.events(), [[0, 2.1, 0, 0, -1, -1, 0, 0]], 1.0)[0]
    assert out[F["termination"]] == O.SINGULARITY


def test_schwarzschild_frequency_ratio_matches_the_circular_orbit_closed_form():
    s, out = O.surface_observable(1.0, 0, 0, 0, 6.0, 20.0, [0, 6, 0, 0, -1, 0, 0, 0])
    assert s == 1
    assert abs(out[2] - math.sqrt(0.5)) <= 4 * EPS


def test_null_circular_limit_is_not_clamped_into_a_timelike_emitter():
    s, _ = O.surface_observable(1.0, 0, 0, 0, 3.0, 3.0, [0, 3, 0, 0, -1, 0, 0, 0])
    assert s == -4  # CircularOrbitIsNotTimelike


@pytest.mark.parametrize("a,q", [(0.0, 0.0), (0.5, 0.0), (0.9, 0.0), (0.998, 0.0), (0.9, 0.3), (0.0, 0.6), (0.6, 0.7)])
def test_prograde_isco_is_the_minimum_of_the_circular_orbit_energy(a, q):
    """The ISCO root (new oracle code) equals the minimum of E(r) along prograde circular orbits."""
    r_isco = O.prograde_isco(1.0, a, q)

    def energy(r):
        k = math.sqrt(r - q * q)
        return (r * r - 2 * r + q * q + a * k) / (r * math.sqrt(r * r - 3 * r + 2 * q * q + 2 * a * k))

    lo, hi = r_isco * 0.9, r_isco * 1.1
    for _ in range(200):  # golden-section search for the minimum
        m1, m2 = lo + 0.382 * (hi - lo), lo + 0.618 * (hi - lo)
        if energy(m1) < energy(m2):
            hi = m2
        else:
            lo = m1
    assert abs(0.5 * (lo + hi) - r_isco) <= 1e-6 * r_isco
    if q == 0.0 and a == 0.0:
        assert abs(r_isco - 6.0) <= 1e-12


def test_ordered_batch_preserves_input_order(golden):
    fx = golden["schwarzschild-scatter-b6-v1"]
    base = np.array(fixture_state(fx))
    states = np.array([base, base * [1, 1, 1, 1, 1, 1, 0.5, 1]])
    states[1, 5] = -math.sqrt(1 - states[1, 6] ** 2 / (1 - 2 / 50.0)) * 0 + base[5]
    one = O.trace_states(1.0, 0, 0, 0, O.regular_v1(), fixture_events(fx), states, 1.0, threads=1)
    two = O.trace_states(1.0, 0, 0, 0, O.regular_v1(), fixture_events(fx), states, 1.0, threads=2)
    np.testing.assert_array_equal(np.nan_to_num(one, nan=-7), np.nan_to_num(two, nan=-7))


def test_both_charts_pull_back_to_the_boyer_lindquist_kerr_newman_metric():
    """The reference's property test (crates/gravlume-domain/src/spacetime.rs:780-878), over 128
    seeded cases: the Kerr-Schild metric of either chart, paired with the Boyer-Lindquist coordinate
    basis written in that chart's Cartesian components, equals the closed-form BL metric within
    128 eps times the pairing's term norm."""
    rng = np.random.default_rng(780)
    eps = np.finfo(float).eps
    for _ in range(128):
        mass = rng.uniform(0.5, 4.0)
        spin, charge = mass * rng.uniform(-0.9, 0.9), mass * rng.uniform(-0.2, 0.2)
        radius = mass * rng.uniform(3.0, 20.0)
        polar, azimuth = rng.uniform(0.1, math.pi - 0.1), rng.uniform(-math.pi, math.pi)
        st, ct = math.sin(polar), math.cos(polar)
        sp, cp = math.sin(azimuth), math.cos(azimuth)
        s2 = st * st
        sigma = radius * radius + spin * spin * ct * ct
        delta = radius * radius - 2.0 * mass * radius + spin * spin + charge * charge
        num = 2.0 * mass * radius - charge * charge
        rf = radius * radius + spin * spin
        expected = np.array([[-1.0 + num / sigma, 0, 0, -num * spin * s2 / sigma],
                             [0, sigma / delta, 0, 0],
                             [0, 0, sigma, 0],
                             [-num * spin * s2 / sigma, 0, 0, s2 * (rf * rf - spin * spin * delta * s2) / sigma]])
        for chart, branch in ((0, 1.0), (1, -1.0)):
            x, y, z = O.oblate_to_cartesian(spin / mass, chart, radius / mass, polar, azimuth)
            x, y, z = x * mass, y * mass, z * mass
            g = O.metric_covariant(mass, spin, charge, chart, [0.0, x, y, z])
            assert g is not None
            cs = branch * spin
            basis = np.array([[1.0, 0, 0, 0],
                              [0, st * cp, st * sp, ct],
                              [0, ct * (radius * cp - cs * sp), ct * (radius * sp + cs * cp), -radius * st],
                              [0, -y, x, 0]])
            basis[1] = basis[1] + branch * ((num / delta) * basis[0] + (spin / delta) * basis[3])
            for r in range(4):
                for c in range(4):
                    terms = g * np.outer(basis[r], basis[c])
                    scale = max(np.abs(terms).sum(), abs(expected[r, c]), 1.0)
                    assert abs(terms.sum() - expected[r, c]) <= 128 * eps * scale, (chart, spin, r, c)
