"""glc_trace_static_scratch (the trace entry point that allocates no device memory) against
glc_trace, called through the C ABI on two jobs in a row.

The no-allocation entry point runs the persistent work-queue kernel out of a static device array;
glc_trace runs the same per-ray arithmetic from its context's allocated job table. Each job is
checked against glc_trace with the binary64 image budget of the parity tests (classes and step
counts exactly, observables within 1e-12 relative). The second job is a different frame and
precision, so it also shows that the shared array's job table and queue counter are rewritten and
cleared between calls. This file sorts last so it runs after the other GPU tests, and it needs
nothing from them when run alone.
"""

import ctypes

import numpy as np
import pytest
import torch

import gravlume_b200 as G
from gravlume_b200 import _native as N
from gravlume_b200.trace import TraceResults, image_camera, raylist_camera
from gpu_common import config1_observation

pytestmark = pytest.mark.gpu

REL = 1e-12


def _job(obs, n_list):
    """One scene with two cameras: its pinhole image and a ray list of n_list of its pixels' states,
    written behind the image in the result arrays."""
    sc = obs.pack()
    w, h = obs.width, obs.height
    cams = [image_camera(0, w, h)]
    states = None
    if n_list:
        from oracle import initial_rays, scene as oracle_scene
        osc = oracle_scene(mass=obs.mass, spin=obs.spin, charge=obs.charge, chart=int(obs.chart),
                           observer_txyz=obs.observer_txyz, target=obs.target_txyz, up_hint=obs.up_hint_xyz,
                           width=w, height=h, vertical_fov=obs.vertical_fov)
        rng = np.random.default_rng(5)
        st, _, _, status = initial_rays(osc, rng.integers(0, w, n_list), rng.integers(0, h, n_list))
        assert (status == 0).all()
        states = torch.tensor(np.asarray(st, dtype=np.float64), device="cuda").contiguous()
        cams.append(raylist_camera(0, states.data_ptr(), n_list, -1.0, offset=w * h))
    return [sc], cams, states, w * h + n_list


def _arrays(scenes, cams):
    return (N.Scene * len(scenes))(*scenes), (N.Camera * len(cams))(*cams)


def _static_trace(scenes, cams, policy, slots):
    res = TraceResults(slots, "cuda")
    sa, ca = _arrays(scenes, cams)
    rs = res.struct()
    stream = torch.cuda.current_stream().cuda_stream
    N.check(N.lib().glc_trace_static_scratch(sa, len(scenes), ca, len(cams), ctypes.byref(policy),
                                             ctypes.byref(rs), ctypes.c_void_p(stream)),
            "glc_trace_static_scratch")
    torch.cuda.synchronize()
    return res.numpy()


def _context_trace(scenes, cams, policy, slots):
    with G.TracePipeline(0, policy) as pipe:
        res = TraceResults(slots, "cuda")
        pipe.trace(scenes, cams, res)
        torch.cuda.synchronize()
        return res.numpy()


def _assert_same(a, b):
    for k in ("termination", "failure", "accepted_steps", "rejected_steps", "radial_turnings",
              "equatorial_crossings", "azimuth_winding", "has_turning_radius"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in ("escape_theta", "escape_phi", "source_radius", "source_azimuth", "frequency_ratio", "travel_time",
              "event_residual", "max_null_residual", "max_lz_drift", "max_carter_drift", "x", "y", "z"):
        x, y = a[k], b[k]
        both = np.isfinite(x) & np.isfinite(y)
        np.testing.assert_array_equal(np.isfinite(x), np.isfinite(y), err_msg=k)
        np.testing.assert_allclose(x[both], y[both], rtol=REL, atol=REL, err_msg=k)


def test_static_scratch_trace_matches_glc_trace_on_two_calls_in_a_row():
    jobs = [
        (config1_observation(width=160, height=96), 64,
         G.ReferencePolicy.frame(G.Precision.FP64, persistent=1)),
        (config1_observation(width=128, height=128, incl_deg=60.0), 0,
         # the no-allocation entry runs MIXED as one kernel (it has no room for hand-off records),
         # so the context path is asked for the same form
         G.ReferencePolicy.frame(G.Precision.MIXED, persistent=1, rays_per_grab=32, refill_interval=2,
                                 mixed_split=0)),
    ]
    for obs, n_list, policy in jobs:
        scenes, cams, keep, slots = _job(obs, n_list)
        got = _static_trace(scenes, cams, policy, slots)
        want = _context_trace(scenes, cams, policy, slots)
        assert (got["termination"] > 0).all()
        _assert_same(got, want)
        del keep


def test_static_scratch_rejects_jobs_beyond_its_capacity():
    obs = config1_observation(width=8, height=8)
    sc = obs.pack()
    scenes = [sc] * 129
    cams = [image_camera(0, 8, 8)]
    sa, ca = _arrays(scenes, cams)
    res = TraceResults(64, "cuda")
    rs = res.struct()
    pol = G.ReferencePolicy.frame(G.Precision.FP32)
    st = N.lib().glc_trace_static_scratch(sa, len(scenes), ca, len(cams), ctypes.byref(pol), ctypes.byref(rs), None)
    assert N.STATUS_NAMES[st] == "CAPACITY"
    assert b"128 scenes" in N.lib().glc_last_error_string()
