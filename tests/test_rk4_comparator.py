"""The second comparator: the reference's own GPU algorithm (the binary32 classical RK4 kernel of
crates/gravlume-render/src/shaders/geodesic_integration.wgsl), restated on the CPU in
oracle/oracle_wgsl_rk4.hpp. It is pinned here by the reference's GPU-against-CPU tests, with their
samples, scenes and tolerances read from the test source into tests/golden/gpu_gate_cases.json:

* the regular matrix (gpu_trace_tests.rs:544-627): the same terminal class as the binary64 CPU
  reference, escape direction within 3.82e-4 rad, event residual within 5e-3, travel time within
  1e-3 M, every drift within the 0.05 budget;
* the surface branch profiles (gpu_trace_tests/surface.rs:232-320): every sample ends on the
  surface in both, with the same radial turnings, equatorial crossings and azimuth winding.
"""

import json
import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O

CASES = json.loads((Path(__file__).parent / "golden" / "gpu_gate_cases.json").read_text())
ANGLE = {"pi/2": math.pi / 2, "pi/3": math.pi / 3, "pi/4": math.pi / 4}


def scene(spin, charge, radius, polar, fov, width, height):
    xyz = O.oblate_to_cartesian(spin, 1, radius, polar, 0.0)
    return O.scene(mass=1.0, spin=spin, charge=charge, chart=1, observer_txyz=(0.0, *xyz), width=width,
                   height=height, vertical_fov=fov)


def test_rk4_comparator_meets_the_reference_regular_matrix_gate():
    c = CASES["regular_matrix"]
    r, polar, _ = c["observer_oblate"]
    sc = scene(c["spin"], c["charge"], r, ANGLE[polar], ANGLE[c["vertical_fov"]], c["width"], c["height"])
    ev = O.events(escape_radius=c["escape_radius"])
    px, py = np.array(c["samples"]).T
    ref, status = O.trace_pixels(sc, O.regular_v1(), ev, px, py)
    assert (status == 0).all()
    gpu = O.rk4_pixels(sc, ev, px, py)
    R = O.RK4
    for i in range(px.size):
        term = int(ref[i, O.F["termination"]])
        assert term in (O.HORIZON, O.ESCAPE)
        assert int(gpu[i, R["termination"]]) == term, (px[i], py[i])
        assert gpu[i, R["flags"]] == 0 and gpu[i, R["steps"]] > 0
        if term == O.ESCAPE:
            d = ref[i, [O.F["escape_dx"], O.F["escape_dy"], O.F["escape_dz"]]]
            g = gpu[i, [R["source0"], R["source1"], R["source2"]]]
            cosine = np.dot(d, g) / (np.linalg.norm(d) * np.linalg.norm(g))
            assert math.acos(min(1.0, cosine)) <= c["escape_angle_rad"]
        assert abs(gpu[i, R["event_residual"]]) <= c["event_residual"]
        assert abs(gpu[i, R["travel_time"]] - ref[i, O.F["travel_time"]]) <= c["travel_time_m"]
        drifts = gpu[i, [R["null_residual"], R["energy_drift"], R["lz_drift"], R["carter_drift"]]]
        assert ((drifts >= 0) & (drifts <= c["drift_limit"])).all()


@pytest.mark.parametrize("profile", CASES["surface_branches"]["profiles"], ids=lambda p: p["label"])
def test_rk4_comparator_meets_the_reference_surface_branch_gate(profile):
    c = CASES["surface_branches"]
    sc = scene(profile["spin"], profile["charge"], profile["observer_radius"], ANGLE[c["observer_polar"]],
               ANGLE[profile["vertical_fov"]], c["width"], c["height"])
    ev = O.events(escape_radius=c["escape_radius"], surface=tuple(c["surface"]))
    px, py = np.array(profile["samples"]).T
    ref, status = O.trace_pixels(sc, O.regular_v1(), ev, px, py)
    assert (status == 0).all()
    gpu = O.rk4_pixels(sc, ev, px, py)
    R = O.RK4
    assert (ref[:, O.F["termination"]] == O.SURFACE).all()
    assert (gpu[:, R["termination"]] == O.SURFACE).all()
    for name in ("radial_turnings", "equatorial_crossings", "azimuth_winding"):
        np.testing.assert_array_equal(gpu[:, R[name]], ref[:, O.F[name]], err_msg=name)
