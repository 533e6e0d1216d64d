"""The batching workload (64 seeded scenes plus a 2048x1024 equirectangular escape map) in one
persistent work-queue launch, replayed as a CUDA graph, and through the autotuner.

Binary64 at rtol 1e-6 (no warp-level precision decisions, so every ray's arithmetic is independent
of which warp traces it): the batch equals per-scene traces of the one-thread-per-ray kernel
(termination classes and step counts on all but a 1e-5 / 1e-4 fraction of rays, floating point to
1e-9 on all but 1e-4 of the rays whose step counts agree: the same code inlined into two kernels may
contract a few FMAs differently, and near-critical rays amplify that rounding); the graph replay equals the direct launch exactly; the autotuned policy
keeps every termination class. A seeded sample of each scene is checked against the binary64 oracle
at the oracle's policy (rtol 1e-10).
"""

import math

import numpy as np
import pytest
import torch

import bench
import gravlume_b200 as G
import oracle as O
from gpu_common import compare

pytestmark = pytest.mark.gpu

INT_FIELDS = ("termination", "failure", "accepted_steps", "rejected_steps", "radial_turnings",
              "equatorial_crossings", "azimuth_winding")
FLOAT_FIELDS = ("escape_theta", "escape_phi", "source_radius", "frequency_ratio", "travel_time", "x", "y", "z")


@pytest.fixture(scope="module")
def job():
    return bench.batch_job(G)


@pytest.fixture(scope="module")
def pipe():
    p = G.TracePipeline(0)
    yield p
    p.close()


def frame64(**kw):
    return G.ReferencePolicy.frame(G.Precision.FP64, position_rtol=1e-6, momentum_rtol=1e-6, position_atol=1e-8,
                                   momentum_atol=1e-8, maximum_step=1000.0, **kw)


def trace(pipe, scenes, cams, slots):
    res = G.TraceResults(slots, "cuda")
    pipe.trace(scenes, cams, res)
    torch.cuda.synchronize()
    return res.numpy()


def assert_same(a, b, sl, exact=False):
    if exact:
        for k in INT_FIELDS + FLOAT_FIELDS:
            np.testing.assert_array_equal(a[k][sl], b[k], err_msg=k)
        return
    # the same per-ray code compiled into two kernels may contract a few FMAs differently; the
    # rounding differences grow along the trace and can, very rarely, flip an accept/reject decision
    n = b["termination"].size
    assert np.count_nonzero(a["termination"][sl] != b["termination"]) <= max(1, n // 100000)
    same = a["accepted_steps"][sl] == b["accepted_steps"]
    assert np.count_nonzero(~same) <= max(1, n // 10000)
    for k in FLOAT_FIELDS:
        # near-critical rays amplify rounding differences exponentially along the trace
        close = np.isclose(a[k][sl][same], b[k][same], rtol=1e-9, atol=1e-9, equal_nan=True)
        assert np.count_nonzero(~close) <= max(1, n // 10000), (k, np.count_nonzero(~close))


def test_one_persistent_launch_equals_per_scene_traces(pipe, job):
    scenes, cams, slots, meta = job
    assert len(scenes) == 65 and slots > 20_000_000
    pipe.set_policy(frame64(persistent=1))
    batch = trace(pipe, scenes, cams, slots)
    assert np.all(batch["termination"] > 0), "every pixel of every camera is written"
    assert (np.bincount(batch["termination"], minlength=9)[[4, 5, 8]] == 0).all()
    pipe.set_policy(frame64(persistent=0))
    for i in (0, 17, 40, 63, 64):
        cam = G.image_camera(0, cams[i].width, cams[i].height, kind=cams[i].kind)
        one = trace(pipe, [scenes[i]], [cam], cams[i].width * cams[i].height)
        sl = slice(cams[i].result_offset, cams[i].result_offset + cams[i].width * cams[i].height)
        assert_same(batch, one, sl)


def test_graph_replay_equals_the_direct_launch(pipe, job):
    scenes, cams, slots, _ = job
    pipe.set_policy(frame64(persistent=1))
    direct = trace(pipe, scenes, cams, slots)
    stream = torch.cuda.Stream()
    res = G.TraceResults(slots, "cuda")
    torch.cuda.synchronize()  # the buffers are initialised on the default stream; the graph runs on another
    graph = pipe.capture_graph(scenes, cams, res, stream)
    for _ in range(2):
        graph.launch(stream)
    stream.synchronize()
    replay = res.numpy()
    graph.close()
    assert_same(direct, replay, slice(None), exact=True)


def test_autotuned_policy_keeps_every_class(pipe, job):
    scenes, cams, slots, _ = job
    sub = [0, 1, 2, 3]
    sc = [scenes[i] for i in sub]
    cm, off = [], 0
    for j, i in enumerate(sub):
        cm.append(G.image_camera(j, cams[i].width, cams[i].height, offset=off))
        off += cams[i].width * cams[i].height
    pipe.set_policy(frame64(persistent=1))
    before = trace(pipe, sc, cm, off)
    tuned = pipe.autotune(sc, cm, repeats=1)
    assert tuned.block_threads % 32 == 0 and tuned.tile_w * tuned.tile_h >= 1
    after = trace(pipe, sc, cm, off)
    np.testing.assert_array_equal(before["termination"], after["termination"])
    np.testing.assert_allclose(before["travel_time"], after["travel_time"], rtol=1e-12, atol=1e-12, equal_nan=True)


def test_batch_sample_matches_the_oracle(pipe, job):
    scenes, cams, slots, meta = job
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, persistent=1))
    rng = np.random.default_rng(9)
    picks = [0, 9, 21, 33, 50, 62]
    for i in picks:
        m = meta[i]
        w = cams[i].width
        osc = O.scene(mass=1.0, spin=m["spin"], charge=m["charge"], chart=1,
                      observer_txyz=list(scenes[i].observer_txyz), width=w, height=w,
                      vertical_fov=math.radians(bench.FOV_DEG))
        ev = O.events(escape_radius=scenes[i].escape_radius, surface=(scenes[i].surface_inner, scenes[i].surface_outer),
                      horizon_offset=1e-3)
        px, py = rng.integers(0, w, 24), rng.integers(0, w, 24)
        ref, status = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, px, py, threads=O.hardware_threads())
        assert (status == 0).all()
        cam = G.image_camera(0, w, w)
        d = trace(pipe, [scenes[i]], [cam], w * w)
        rep = compare(d, py * w + px, ref)
        print(i, m, rep)
        assert rep["class_mismatch"] == 0, (i, rep)
        if "travel_time" in rep:
            assert rep["travel_time"] <= 1e-6 * max(1.0, m["observer_radius"]), (i, rep)


@pytest.mark.parametrize("persistent", [1, 2])
def test_mixed_work_queue_kernels_run_the_two_kernel_form(pipe, job, persistent):
    """MIXED through the lane-refill and the warp-grab work queues: the binary32 bulk stepping runs
    in the queue kernel and the binary64 completion after it, and every ray ends as it does in the
    one-thread-per-ray launch. The lane-refill kernel inlines the binary32 step into other code, and
    binary32 contractions that round differently flip accept/reject decisions of steps whose error
    estimate sits at the tolerance (about 2 % of the rays take another step sequence), so the
    observables are compared at the frame tolerance's truncation level."""
    scenes, cams, slots, _ = job
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, persistent=0))
    simple = trace(pipe, scenes, cams, slots)
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, persistent=persistent))
    queued = trace(pipe, scenes, cams, slots)
    assert pipe.stats().last_persistent == persistent
    assert np.all(queued["f64_steps"][queued["flags"] & 0x30 == 0] >= 1), "every integrated ray was completed"
    # every ray of the batch ends by an event: none may run to the step or reject caps, which is
    # what a completion that misses the event the bulk kernel handed over for would do
    for d in (simple, queued):
        assert not np.any(np.isin(d["termination"], [G.Termination.STEP_EXHAUSTION, G.Termination.REJECT_EXHAUSTION]))
    steps = lambda d: d["accepted_steps"].astype(np.int64) + d["rejected_steps"]
    assert steps(queued).max() <= 2 * steps(simple).max()
    n = slots
    assert np.count_nonzero(queued["termination"] != simple["termination"]) <= max(1, n // 100000)
    same = queued["termination"] == simple["termination"]
    for k in ("escape_theta", "escape_phi", "frequency_ratio", "source_radius"):
        a, b = queued[k][same], simple[k][same]
        close = np.isclose(a, b, rtol=1e-4, atol=1e-4, equal_nan=True)
        assert np.count_nonzero(~close) <= max(1, n // 10000), (k, np.count_nonzero(~close))
