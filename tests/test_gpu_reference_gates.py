"""The reference's own GPU contract gates (crates/gravlume-render/src/gpu_trace_tests.rs), on the
CUDA path and against the binary64 oracle:

- event ties by affine distance and stable protocol order (:233-269), and surface-event arming
  that needs the value to leave the profile band (:271-294): the reference's synthetic cases
  (shaders/event_policy_capture.wgsl) run by the kernels' own selection and arming functions;
- the mass scale does not change the dimensionless result (:296-308): bitwise;
- the coordinate-time origin does not change the observables (:310-345): bitwise;
- every recorded invariant can make a terminal Uncertain (:380-392), with the replaced kernel's
  gate switched on (policy.uncertain_terminals);
- the accelerated sky (escape-direction map) keeps the full trace's terminals and its escape
  directions within 3.82e-4 rad on the reference's four transfer profiles (:630-697), checked
  against the oracle's own rays as well as against the full CUDA trace;
- an adjacent shadow-edge pair matches the oracle's classification (:700-750), and so do the
  refinement's four subpixel samples of the edge pixels."""

import math

import numpy as np
import pytest
import torch

import gravlume_b200 as G
from gravlume_b200 import _native as N
import oracle as O
from gpu_common import oracle_for, seeded_pixels, unit

pytestmark = pytest.mark.gpu

H_, S_, E_ = 1 << 1, 1 << 2, 1 << 3  # candidate bits: horizon, surface, escape


def reference_observation(width, height, mass=1.0, spin=0.8, charge=0.0, r_obs=30.0, fov=math.pi / 4, t0=0.0,
                          escape=200.0):
    """default_observation / observation_at_scale / observation_at_coordinate_time / transfer_profile
    of the reference's tests: observer at oblate radius r_obs and polar angle pi/3, looking at the
    origin with up (0, 0, 1), escape sphere at 200 M, no surface."""
    xyz = G.oblate_to_cartesian(spin * mass, G.KerrSchildChart.OUTGOING, r_obs * mass, math.pi / 3, 0.0)
    return G.Observation(mass=mass, spin=spin * mass, charge=charge * mass, chart=G.KerrSchildChart.OUTGOING,
                         observer_txyz=(t0, *xyz), target_txyz=(t0, 0.0, 0.0, 0.0), width=width, height=height,
                         vertical_fov=fov, escape_radius=escape * mass)


def trace_bytes(pipe, obs):
    res = pipe.trace([obs.pack()], [G.image_camera(0, obs.width, obs.height)])
    torch.cuda.synchronize()
    return {k: v.cpu().numpy().copy() for k, v in res.buffers.items()}, res.numpy()


@pytest.mark.parametrize("preset", ["regular_v1", "frame_mixed"])
def test_event_ties_and_surface_arming_follow_the_reference_cases(preset):
    pol = G.ReferencePolicy.regular_v1() if preset == "regular_v1" else G.ReferencePolicy.frame(G.Precision.MIXED)
    out = torch.zeros((8, 4), dtype=torch.int32, device="cuda")
    N.check(N.lib().glc_selftest_event_policy(pol, out.data_ptr(), None), "glc_selftest_event_policy")
    torch.cuda.synchronize()
    got = out.cpu().numpy().astype(np.int64)
    T = G.Termination
    want = [(T.ESCAPE, S_ | E_), (T.ESCAPE, S_ | E_), (T.EQUATORIAL_SURFACE, S_ | E_),
            (T.EQUATORIAL_SURFACE, H_ | S_)]
    for case, (term, cand) in enumerate(want):
        assert tuple(got[case, :3]) == (int(term), cand, 1), (case, got[case])
    assert list(got[4:, 0]) == [0, 0, 1, 1], "surface, in-band, outside-band and sticky-armed cases"


@pytest.mark.parametrize("precision", [G.Precision.FP32, G.Precision.MIXED, G.Precision.FP64])
def test_mass_scale_does_not_change_the_dimensionless_result(precision):
    with G.TracePipeline(0, G.ReferencePolicy.frame(precision)) as pipe:
        unit_, d = trace_bytes(pipe, reference_observation(7, 5, mass=1.0))
        scaled, _ = trace_bytes(pipe, reference_observation(7, 5, mass=8.0))
    for k in unit_:
        np.testing.assert_array_equal(unit_[k], scaled[k], err_msg=k)
    # and the classes are the oracle's
    obs = reference_observation(7, 5)
    osc, ev, _ = oracle_for(obs)
    idx = np.arange(35)
    ref, _ = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, idx % 7, idx // 7, threads=O.hardware_threads())
    np.testing.assert_array_equal(d["termination"], ref[:, O.F["termination"]].astype(int))


def test_coordinate_time_origin_does_not_change_the_observables():
    with G.TracePipeline(0, G.ReferencePolicy.frame(G.Precision.MIXED)) as pipe:
        origin, d = trace_bytes(pipe, reference_observation(7, 5, t0=0.0))
        translated, _ = trace_bytes(pipe, reference_observation(7, 5, t0=1.0e8))
    assert d["termination"][0] == G.Termination.ESCAPE
    for k in origin:
        np.testing.assert_array_equal(origin[k], translated[k], err_msg=k)


def test_recorded_invariant_drift_can_make_a_terminal_uncertain():
    obs = reference_observation(64, 36)
    with G.TracePipeline(0) as pipe:
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64))
        _, plain = trace_bytes(pipe, obs)
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, uncertain_terminals=1))
        _, gated = trace_bytes(pipe, obs)
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, uncertain_terminals=1,
                                                uncertain_drift_limit=1e-300))
        _, tiny = trace_bytes(pipe, obs)
    # the reference budget leaves this view's terminals alone; a zero budget gates every event terminal
    np.testing.assert_array_equal(gated["termination"], plain["termination"])
    events = np.isin(plain["termination"], [G.Termination.HORIZON_CROSSING, G.Termination.ESCAPE])
    drifted = (plain["max_null_residual"] > 0) | (plain["max_lz_drift"] > 0) | (plain["max_carter_drift"] > 0)
    assert (events & drifted).sum() > 0.9 * events.sum()
    assert np.all(tiny["termination"][events & drifted] == G.Termination.UNCERTAIN)
    assert np.all(tiny["termination"][~events] == plain["termination"][~events])


TRANSFER_PROFILES = [("default", 0.8, 0.0, 30.0, math.pi / 4), ("near-extreme-wide", 0.99, 0.0, 30.0, math.pi / 2),
                     ("negative-near", -0.8, 0.0, 5.0, math.pi / 4), ("kerr-newman", 0.6, 0.5, 30.0, math.pi / 4)]


@pytest.mark.parametrize("label,spin,charge,r_obs,fov", TRANSFER_PROFILES)
def test_accelerated_sky_keeps_terminals_and_directions_against_the_oracle(label, spin, charge, r_obs, fov):
    w, h = 1280, 720
    obs = reference_observation(w, h, spin=spin, charge=charge, r_obs=r_obs, fov=fov)
    pol = dict(position_rtol=1e-8, momentum_rtol=1e-8, position_atol=1e-10, momentum_atol=1e-10, maximum_step=1e3)
    with G.TracePipeline(0) as pipe:
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, **pol))
        _, full = trace_bytes(pipe, obs)
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, escape_map=1, **pol))
        _, acc = trace_bytes(pipe, obs)
    np.testing.assert_array_equal(acc["termination"], full["termination"], err_msg=label)
    np.testing.assert_array_equal(acc["candidates"], full["candidates"], err_msg=label)
    rec = np.flatnonzero((acc["flags"] & 32) != 0)
    if r_obs >= 30.0:
        assert rec.size > 0, f"{label}: the far-field view did not exercise the escape-direction map"
    if rec.size == 0:
        return
    # the oracle's own rays for a seeded sample of the reconstructed pixels
    rng = np.random.default_rng(697)
    pick = np.sort(rng.choice(rec, size=min(256, rec.size), replace=False))
    osc, ev, _ = oracle_for(obs)
    ref, _ = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, pick % w, pick // w, threads=O.hardware_threads())
    assert np.all(ref[:, O.F["termination"]].astype(int) == G.Termination.ESCAPE), label
    d = np.stack([ref[:, O.F["escape_dx"]], ref[:, O.F["escape_dy"]], ref[:, O.F["escape_dz"]]], axis=1)
    v = unit(acc["escape_theta"][pick], acc["escape_phi"][pick])
    chord = np.linalg.norm(d - v, axis=1)
    print(label, "reconstructed", rec.size, "max chord vs oracle", float(chord.max()))
    assert chord.max() <= 3.82e-4, label


def test_shadow_edge_pairs_and_refinement_samples_match_the_oracle():
    w, h = 160, 90
    obs = reference_observation(w, h)
    sc = obs.pack()
    cam = [G.image_camera(0, w, h)]
    with G.TracePipeline(0, G.ReferencePolicy.frame(G.Precision.FP64)) as pipe:
        primary = G.TraceResults(w * h, "cuda")
        pipe.trace([sc], cam, primary)
        cov = pipe.refine_shadow_edges([sc], cam, primary).cpu().numpy()
        torch.cuda.synchronize()
        d = primary.numpy()
    t = d["termination"].reshape(h, w)
    osc, ev, _ = oracle_for(obs)
    pol = O.custom_policy(1e-10, 1e-12)
    threads = O.hardware_threads()
    # every horizontally adjacent horizon/escape pair: both pixels classified as the oracle does
    left = np.argwhere(np.isin(t[:, :-1], [1, 2]) & np.isin(t[:, 1:], [1, 2]) & (t[:, :-1] != t[:, 1:]))
    assert len(left) > 0, "the default view has a horizontal horizon/escape boundary"
    py = np.concatenate([left[:, 0], left[:, 0]])
    px = np.concatenate([left[:, 1], left[:, 1] + 1])
    ref, _ = O.trace_pixels(osc, pol, ev, px, py, threads=threads)
    np.testing.assert_array_equal(t[py, px], ref[:, O.F["termination"]].astype(int))
    # the refinement's four rotated-grid subpixel samples of each refined pixel, by the oracle
    c = cov.reshape(h, w)
    ey, ex = np.nonzero((c > 0) & (c < 1) | (np.isin(c, [0.0, 1.0]) & edge_mask(t)))
    esc = np.zeros(ey.size)
    for ox, oy in [(0.375, 0.125), (0.875, 0.375), (0.625, 0.875), (0.125, 0.625)]:
        r, _ = O.trace_pixels(osc, pol, ev, ex, ey, ox, oy, threads=threads)
        esc += r[:, O.F["termination"]].astype(int) == G.Termination.ESCAPE
    mism = np.count_nonzero(c[ey, ex] != 0.25 * esc)
    print("refined pixels", ey.size, "coverage differing from the oracle's samples", mism)
    assert ey.size > 50
    assert mism <= max(1, ey.size // 100), mism


def edge_mask(t):
    """Capture/escape pixels with a 4-neighbour of the other class."""
    b = np.where(t == 1, 0, np.where(t == 2, 1, -1))
    h, w = b.shape
    edge = np.zeros((h, w), bool)
    for dy, dx in ((0, 1), (0, -1), (1, 0), (-1, 0)):
        nb = np.full((h, w), -2)
        ys, xs = slice(max(dy, 0), h + min(dy, 0)), slice(max(dx, 0), w + min(dx, 0))
        yd, xd = slice(max(-dy, 0), h + min(-dy, 0)), slice(max(-dx, 0), w + min(-dx, 0))
        nb[yd, xd] = b[ys, xs]
        edge |= (b >= 0) & (nb == 1 - b)
    return edge
