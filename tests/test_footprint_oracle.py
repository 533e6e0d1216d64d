"""The oracle's surface footprint (oracle/oracle_footprint.hpp) against the reference's own footprint
tests: the canonical blackbody/bolometric surface sample is resolved with one exact branch key
(surface_observable_tests.rs:76-110), a stencil that leaves the pixel is rejected (112-133), and the
singular values keep every binary minor axis bit-exactly (footprint.rs:270-291). A row across the
disk's edge shows the resolved/discontinuity/no-surface split the GPU kernels must reproduce."""

import json
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from test_oracle_fixtures import default_observation_scene

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_fixtures.json").read_text())


def canonical():
    base = GOLDEN["kerr-exterior-observation-v1"]
    fx = GOLDEN["kerr-equatorial-surface-observable-v1"]
    sc = default_observation_scene(base)
    s = fx["surface"]
    ev = O.events(escape_radius=200.0, surface=(float(s["inner_radius_m"]), float(s["outer_radius_m"])))
    return sc, ev, fx["sample"]["x"], fx["sample"]["y"]


def test_canonical_surface_footprint_is_resolved_with_one_exact_branch_key():
    sc, ev, x, y = canonical()
    out, status = O.surface_footprint(sc, O.regular_v1(), ev, [x], [y])
    assert status[0] == 1
    j, (major, minor), parity = out[0, :4], out[0, 4:6], out[0, 7]
    assert np.all(np.isfinite(j))
    assert major >= minor > 0.0
    assert parity != 0.0
    # the terminal surface crossing is not part of the branch key
    row, _ = O.trace_pixels(sc, O.regular_v1(), ev, [x], [y])
    assert row[0, O.F["equatorial_crossings"]] == 0
    # the Jacobian is the central difference of the neighbours' anchors
    off = [(-0.25, 0.0), (0.25, 0.0), (0.0, -0.25), (0.0, 0.25)]
    nb = [O.trace_pixels(sc, O.regular_v1(), ev, [x], [y], 0.5 + dx, 0.5 + dy)[0][0] for dx, dy in off]
    rc, pc = row[0, O.F["source_radius"]], row[0, O.F["source_azimuth"]]
    arc = [rc * ((n[O.F["source_azimuth"]] - pc + np.pi) % (2 * np.pi) - np.pi) for n in nb]
    r = [n[O.F["source_radius"]] for n in nb]
    want = [(r[1] - r[0]) / 0.5, (r[3] - r[2]) / 0.5, (arc[1] - arc[0]) / 0.5, (arc[3] - arc[2]) / 0.5]
    np.testing.assert_allclose(j, want, rtol=1e-12, atol=1e-15)


def test_footprint_rejects_a_neighbourhood_outside_one_pixel():
    sc, ev, x, y = canonical()
    with pytest.raises(ValueError, match=r"\[0.25, 0.75\]"):
        O.surface_footprint(sc, O.regular_v1(), ev, [x], [y], 0.125, 0.5)


@pytest.mark.parametrize("exponent", [-1074, -1022, -700, -52, -1, 0])
def test_determinant_quotient_preserves_every_binary_singular_axis(exponent):
    minor = 2.0 ** exponent
    m = O.footprint_metrics([1.0, 0.0, 0.0, minor])
    assert m is not None
    assert m[2] == 1.0 and m[3] == minor
    assert O.footprint_metrics([1.0, np.nan, 0.0, 1.0]) is None


def test_row_across_the_disk_edge_splits_into_the_three_outcomes():
    sc, ev, _, _ = canonical()
    xs = np.array([600, 606, 608, 640, 716, 718])
    out, status = O.surface_footprint(sc, O.regular_v1(), ev, xs, np.full(xs.size, 16), threads=O.default_threads())
    assert status.tolist() == [0, 2, 2, 1, 2, 0]
    assert np.all(np.isnan(out[status != 1]))
    res = out[status == 1]
    assert np.all(res[:, 4] >= res[:, 5])
    # |det| = major * minor
    np.testing.assert_allclose(np.abs(res[:, 6]), res[:, 4] * res[:, 5], rtol=1e-14)
