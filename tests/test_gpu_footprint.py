"""Surface footprint on the GPU (glc_surface_footprint; footprint.rs:74-235).

- The quarter-pixel method is the reference's estimate: at the canonical surface sample and on
  seeded pixels of the a=0.9, Q=0.3 frame its status, Jacobian, singular values and parity match
  the oracle's restatement traced with the same binary64 policy (Jacobian within 1e-7 of its
  largest component: both sides difference the same adaptive integrations, rounded by different
  compilers). Up to 1 % of the pixels may change status, where a neighbour's branch flips between
  the two integrations.
- The tangent method is the derivative of the computed trace: it agrees with central differences of
  full frames traced a 1/64 pixel apart at a tight binary64 tolerance (pinhole and equirectangular
  cameras), and with the reference's quarter-pixel estimate at the canonical sample to the reference
  GPU test's own 3e-3 of the largest component (gpu_trace_tests/surface.rs:69-118). In binary32 and
  MIXED it stays within 1e-4 of the binary64 tangent on 99 % of the pixels.
"""

import math

import numpy as np
import pytest
import torch

import gravlume_b200 as G
import oracle as O
from gpu_common import config1_observation, oracle_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pipe():
    p = G.TracePipeline(0)
    yield p
    p.close()


def canonical_observation(golden):
    base = golden["kerr-exterior-observation-v1"]
    return G.Observation.from_oblate(float(base["observer"]["oblate_radius_m"]),
                                     float(base["observer"]["polar_angle_rad"]), 0.0, spin=0.8,
                                     chart=G.KerrSchildChart.INGOING, width=1280, height=720,
                                     vertical_fov=float(base["viewport"]["vertical_fov_rad"]), escape_radius=200.0,
                                     surface=G.EquatorialSurface(6.0, 20.0, 1.0))


def footprint(pipe, obs, method, subpixel=(0.5, 0.5), kind=G._native.CAMERA_PINHOLE, size=None):
    sc = obs.packed
    w, h = size or (sc.width, sc.height)
    cam = [G.image_camera(0, w, h, subpixel, kind=kind)]
    primary = G.TraceResults(w * h, "cuda")
    pipe.trace([sc], cam, primary)
    fp = pipe.surface_footprint([sc], cam, primary, method)
    torch.cuda.synchronize()
    return G.footprint_fields(fp), primary.numpy()


def frame(pipe, obs, subpixel, kind=G._native.CAMERA_PINHOLE, size=None):
    sc = obs.packed
    w, h = size or (sc.width, sc.height)
    d = pipe.trace([sc], [G.image_camera(0, w, h, subpixel, kind=kind)]).numpy()
    torch.cuda.synchronize()
    return d


def max_component_error(a, b):
    """Per-pixel max |a - b| over the four components, relative to max |b| (the reference's measure)."""
    a, b = np.asarray(a).reshape(-1, 4), np.asarray(b).reshape(-1, 4)
    return np.max(np.abs(a - b), axis=1) / np.max(np.abs(b), axis=1)


def test_canonical_sample_matches_the_oracle_and_the_tangent(pipe, golden):
    obs = canonical_observation(golden)
    osc, ev, _ = oracle_for(obs)
    fx = golden["kerr-equatorial-surface-observable-v1"]["sample"]
    xs = np.array([600, 606, 608, fx["x"], 716, 718])
    ref, rstat = O.surface_footprint(osc, O.regular_v1(), ev, xs, np.full(xs.size, fx["y"]),
                                     threads=O.default_threads())
    assert rstat.tolist() == [0, 2, 2, 1, 2, 0]
    pipe.set_policy(G.ReferencePolicy.regular_v1())
    q, d = footprint(pipe, obs, "quarter_pixel")
    t, _ = footprint(pipe, obs, "tangent")
    sel = fx["y"] * 1280 + xs
    assert q["status"][sel].tolist() == rstat.tolist()
    i = fx["y"] * 1280 + fx["x"]
    want = ref[3]
    assert max_component_error(q["jacobian"][i], want[:4])[0] <= 1e-7
    np.testing.assert_allclose(q["singular_values"][i], want[4:6], rtol=1e-6)
    assert q["parity"][i] == want[7] != 0
    assert q["singular_values"][i, 0] >= q["singular_values"][i, 1] > 0
    assert d["equatorial_crossings"][i] == 0
    # the tangent against the reference estimate, at the reference GPU test's tolerance
    assert t["status"][i] == G.FootprintStatus.RESOLVED
    assert max_component_error(t["jacobian"][i], want[:4])[0] <= 3e-3
    assert t["parity"][i] == want[7]
    # every non-resolved entry is NaN; NO_SURFACE exactly where the center is not a surface hit
    for f in (q, t):
        bad = f["status"] != G.FootprintStatus.RESOLVED
        assert np.all(np.isnan(f["jacobian"][bad]))
        c = d["candidates"]
        hit = (d["termination"] == G.Termination.EQUATORIAL_SURFACE) & ((d["flags"] & 4) == 0) & ((c & (c - 1)) == 0)
        assert np.all((f["status"] == G.FootprintStatus.NO_SURFACE) == ~hit)


def test_quarter_pixel_matches_the_oracle_on_seeded_pixels(pipe):
    obs = config1_observation()
    osc, ev, _ = oracle_for(obs)
    pipe.set_policy(G.ReferencePolicy.regular_v1())
    q, d = footprint(pipe, obs, "quarter_pixel")
    # sample among the surface pixels of the frame, plus a band of every status
    surf = np.flatnonzero(d["termination"] == G.Termination.EQUATORIAL_SURFACE)
    rng = np.random.default_rng(7)
    idx = np.sort(np.concatenate([rng.choice(surf, 240, replace=False),
                                  np.flatnonzero(q["status"] == G.FootprintStatus.DISCONTINUITY)[:60]]))
    idx = np.unique(idx)
    ref, rstat = O.surface_footprint(osc, O.regular_v1(), ev, idx % 256, idx // 256, threads=O.default_threads())
    gst = q["status"][idx]
    same = gst == rstat
    print("statuses", np.bincount(rstat, minlength=4), "mismatches", int((~same).sum()))
    assert (~same).sum() <= max(1, idx.size // 100)
    both = same & (rstat == 1)
    assert both.sum() > 150
    err = max_component_error(q["jacobian"][idx][both], ref[both, :4])
    assert err.max() <= 1e-7, err.max()
    np.testing.assert_allclose(q["singular_values"][idx][both], ref[both, 4:6], rtol=1e-6, atol=1e-12)
    assert np.array_equal(q["parity"][idx][both], ref[both, 7].astype(np.int32))


@pytest.mark.parametrize("kind", [G._native.CAMERA_PINHOLE, G._native.CAMERA_EQUIRECT])
def test_tangent_is_the_derivative_of_the_trace(pipe, kind):
    obs = config1_observation()
    size = (256, 256) if kind == G._native.CAMERA_PINHOLE else (512, 256)
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, position_rtol=1e-12, momentum_rtol=1e-12,
                                            position_atol=1e-14, momentum_atol=1e-14, maximum_step=1000.0))
    t, d = footprint(pipe, obs, "tangent", kind=kind, size=size)
    ok = t["status"] == G.FootprintStatus.RESOLVED
    assert ok.sum() > 1000
    delta = 1.0 / 64.0
    nb = [frame(pipe, obs, s, kind, size) for s in ((0.5 - delta, 0.5), (0.5 + delta, 0.5), (0.5, 0.5 - delta),
                                                     (0.5, 0.5 + delta))]
    same = ok.copy()
    for n in nb:
        same &= (n["termination"] == G.Termination.EQUATORIAL_SURFACE) & (
            n["radial_turnings"] == d["radial_turnings"]) & (n["azimuth_winding"] == d["azimuth_winding"])
    rc, pc = d["source_radius"], d["source_azimuth"]
    arc = [rc * ((n["source_azimuth"] - pc + math.pi) % (2 * math.pi) - math.pi) for n in nb]
    fd = np.stack([(nb[1]["source_radius"] - nb[0]["source_radius"]) / (2 * delta),
                   (nb[3]["source_radius"] - nb[2]["source_radius"]) / (2 * delta),
                   (arc[1] - arc[0]) / (2 * delta), (arc[3] - arc[2]) / (2 * delta)], axis=1)
    err = max_component_error(t["jacobian"].reshape(-1, 4)[same], fd[same])
    print("pixels", int(same.sum()), "median", float(np.median(err)), "p99", float(np.quantile(err, 0.99)),
          "max", float(err.max()))
    assert np.median(err) <= 1e-5
    assert np.quantile(err, 0.99) <= 1e-4


@pytest.mark.parametrize("precision", [G.Precision.FP32, G.Precision.MIXED])
def test_binary32_tangents_follow_the_binary64_tangent(pipe, precision):
    obs = config1_observation()
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64))
    t64, _ = footprint(pipe, obs, "tangent")
    pipe.set_policy(G.ReferencePolicy.frame(precision))
    t32, _ = footprint(pipe, obs, "tangent")
    ok = (t64["status"] == 1) & (t32["status"] == 1)
    assert ok.sum() > 1000
    err = max_component_error(t32["jacobian"].reshape(-1, 4)[ok], t64["jacobian"].reshape(-1, 4)[ok])
    print(precision.name, "median", float(np.median(err)), "p99", float(np.quantile(err, 0.99)))
    assert np.quantile(err, 0.99) <= 1e-4
    assert np.mean(t32["parity"][ok] == t64["parity"][ok]) >= 0.999


def test_footprint_rejects_ray_lists_and_off_center_stencils(pipe):
    obs = config1_observation(width=32, height=32)
    sc = obs.packed
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64))
    cam = [G.image_camera(0, 32, 32, (0.125, 0.5))]
    primary = G.TraceResults(32 * 32, "cuda")
    pipe.trace([sc], cam, primary)
    with pytest.raises(G.GlcError, match="0.25, 0.75"):
        pipe.surface_footprint([sc], cam, primary, "quarter_pixel")
    # the tangent needs no stencil
    fp = G.footprint_fields(pipe.surface_footprint([sc], cam, primary, "tangent"))
    torch.cuda.synchronize()
    assert set(np.unique(fp["status"])) <= {0, 1}
    states = torch.zeros((4, 8), dtype=torch.float64, device="cuda")
    rl = [G.raylist_camera(0, states.data_ptr(), 4, -1.0)]
    with pytest.raises(G.GlcError, match="image cameras"):
        pipe.surface_footprint([sc], rl, G.TraceResults(4, "cuda"), "tangent")


@pytest.mark.parametrize("method", ["quarter_pixel", "tangent"])
def test_two_cameras_in_one_call_equal_separate_calls(pipe, method):
    """Two image cameras of different scenes and sizes in one call (results at their own offsets)
    give each camera's footprints of a call with that camera alone (binary64: per-ray results do
    not depend on which rays share a warp)."""
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64))
    o1 = config1_observation(width=192, height=160)
    o2 = config1_observation(width=128, height=96, spin=0.5, charge=0.0, incl_deg=60.0)
    sc = [o1.packed, o2.packed]
    n1, n2 = 192 * 160, 128 * 96
    cams = [G.image_camera(0, 192, 160), G.image_camera(1, 128, 96, offset=n1 + 7)]
    primary = G.TraceResults(n1 + 7 + n2, "cuda")
    pipe.trace(sc, cams, primary)
    both = G.footprint_fields(pipe.surface_footprint(sc, cams, primary, method))
    torch.cuda.synchronize()
    for k, (o, cam, off, n) in enumerate(((o1, cams[0], 0, n1), (o2, cams[1], n1 + 7, n2))):
        alone, _ = footprint(pipe, o, method)
        for name in ("jacobian", "singular_values", "determinant", "status", "parity"):
            np.testing.assert_array_equal(both[name][off:off + n], alone[name], err_msg=f"{name} camera {k}")
        assert (alone["status"] == G.FootprintStatus.RESOLVED).sum() > 100
