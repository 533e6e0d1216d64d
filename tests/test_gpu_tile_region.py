"""Tile regions on the trace boundary (TileRegion of the reference's encode_batch,
crates/gravlume-render/src/trace.rs:701-710, 799-857): a frame traced batch by batch, in the
reference renderer's schedule, equals the frame traced at once byte for byte, in every precision
mode, with the escape-direction map and the capture certificates, through glc_trace,
glc_trace_host, a CUDA graph and glc_trace_static_scratch; invalid regions are rejected."""

import ctypes

import numpy as np
import pytest
import torch

import gravlume_b200 as G
from gravlume_b200 import _native as N
from gravlume_b200.batches import TileRegion, TraceProgress
from gravlume_b200.trace import TraceResults, image_camera
from gpu_common import config1_observation

pytestmark = pytest.mark.gpu

W, H = 200, 138  # 25 x 18 tiles, the last row of tiles two pixels high


def _bytes(res: TraceResults) -> dict:
    return {k: v.cpu().numpy().copy() for k, v in res.buffers.items()}


def _assert_equal(a: dict, b: dict):
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("precision,extra", [(G.Precision.FP32, {}), (G.Precision.MIXED, {}),
                                             (G.Precision.MIXED, {"mixed_split": 0}),
                                             (G.Precision.FP64, {})])
def test_batched_frame_equals_the_one_shot_frame(precision, extra):
    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    with G.TracePipeline(0, G.ReferencePolicy.frame(precision, **extra)) as pipe:
        one = pipe.trace([sc], [image_camera(0, W, H)])
        torch.cuda.synchronize()
        # a small initial budget, so that the schedule mixes row runs and whole-row blocks
        res, done = pipe.trace_progressive([sc], image_camera(0, W, H), progress=TraceProgress(W, H, 65535, 11))
        torch.cuda.synchronize()
    assert len(done) > 2
    assert any(b.workgroups[1] == 1 and b.workgroups[0] < 25 for b, _ in done)
    assert done[-1][0].finishes(W, H)
    _assert_equal(_bytes(one), _bytes(res))


def test_batched_sky_with_escape_map_and_certificates_equals_the_one_shot_frame():
    w, h = 520, 300  # 65 x 38 tiles, the last tile row four pixels high
    obs = config1_observation(width=w, height=h, surface=False)
    sc = obs.pack()
    pol = G.ReferencePolicy.frame(G.Precision.MIXED, escape_map=1, capture_certificates=1)
    with G.TracePipeline(0, pol) as pipe:
        one = pipe.trace([sc], [image_camera(0, w, h)])
        torch.cuda.synchronize()
        d = one.numpy()
        assert ((d["flags"] >> 5) & 1).any(), "some tiles are reconstructed from the map"
        assert ((d["flags"] >> 4) & 1).any(), "some tiles are certified captures"
        res, done = pipe.trace_progressive([sc], image_camera(0, w, h), progress=TraceProgress(w, h, 65535, 29))
        torch.cuda.synchronize()
    _assert_equal(_bytes(one), _bytes(res))


def test_a_region_writes_only_its_pixels():
    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    region = TileRegion((3, 2), (5, 4))
    with G.TracePipeline(0, G.ReferencePolicy.frame(G.Precision.FP32)) as pipe:
        res = pipe.trace([sc], [image_camera(0, W, H, region=region)])
        torch.cuda.synchronize()
    code = res.buffers["code"].cpu().numpy().view(np.uint32).reshape(H, W, 4)
    x0, y0, x1, y1 = region.pixel_rect(W, H)
    inside = np.zeros((H, W), dtype=bool)
    inside[y0:y1, x0:x1] = True
    assert np.all(code[inside][:, 0] & 0xFF != 0xFF)  # traced (a termination code)
    assert np.all(code[~inside] == 0xFFFFFFFF)        # untouched fill pattern


def test_batched_host_trace_equals_the_one_shot_host_trace():
    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    with G.TracePipeline(0, G.ReferencePolicy.frame(G.Precision.MIXED)) as pipe:
        a = TraceResults(W * H, None, host=True)
        b = TraceResults(W * H, None, host=True)
        sa, ca = pipe._arrays([sc], [image_camera(0, W, H)])
        N.check(N.lib().glc_trace_host(pipe._h, sa, 1, ca, 1, a.struct()), "glc_trace_host")
        progress = TraceProgress(W, H, 65535, 41)
        while (batch := progress.next_batch()) is not None:
            sa, ca = pipe._arrays([sc], [image_camera(0, W, H, region=batch)])
            N.check(N.lib().glc_trace_host(pipe._h, sa, 1, ca, 1, b.struct()), "glc_trace_host")
            progress.submitted(batch)
            progress.completed(10.0)
    _assert_equal(_bytes(a), _bytes(b))


def test_graph_and_static_scratch_take_regions():
    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    region = TileRegion((0, 5), (25, 3))
    cam = image_camera(0, W, H, region=region)
    pol = G.ReferencePolicy.frame(G.Precision.FP64)
    with G.TracePipeline(0, pol) as pipe:
        want = pipe.trace([sc], [cam])
        torch.cuda.synchronize()
        got_graph = TraceResults(W * H, torch.device("cuda", 0))
        torch.cuda.synchronize()  # the fill of the result arrays precedes the graph's stream
        stream = torch.cuda.Stream()
        with torch.cuda.stream(stream):
            g = pipe.capture_graph([sc], [cam], got_graph, stream=stream)
            g.launch(stream)
        stream.synchronize()
        g.close()
    got_static = TraceResults(W * H, torch.device("cuda", 0))
    sa, ca = G.TracePipeline._arrays([sc], [cam])
    N.check(N.lib().glc_trace_static_scratch(sa, 1, ca, 1, ctypes.byref(pol), ctypes.byref(got_static.struct()),
                                             ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)),
            "glc_trace_static_scratch")
    torch.cuda.synchronize()
    _assert_equal(_bytes(want), _bytes(got_graph))
    _assert_equal(_bytes(want), _bytes(got_static))


def test_invalid_regions_are_rejected():
    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    with G.TracePipeline(0) as pipe:
        res = TraceResults(W * H, torch.device("cuda", 0))
        for origin, count in (((24, 0), (2, 1)), ((0, 17), (1, 2)), ((0, 0), (0, 3))):
            cam = image_camera(0, W, H)
            cam.tile_origin[:] = list(origin)
            cam.tile_count[:] = list(count)
            sa, ca = pipe._arrays([sc], [cam])
            st = N.lib().glc_trace(pipe._h, sa, 1, ca, 1, ctypes.byref(res.struct()), None)
            assert N.STATUS_NAMES[st] == "INVALID_ARGUMENT", (origin, count)
        # whole-view passes reject a region
        one = pipe.trace([sc], [image_camera(0, W, H)])
        cam = image_camera(0, W, H, region=TileRegion((0, 0), (1, 1)))
        with pytest.raises(G.GlcError):
            pipe.refine_shadow_edges([sc], [cam], one)


@pytest.mark.parametrize("world", [2, 3, 4])
def test_rank_bands_traced_one_after_another_reassemble_the_frame(world):
    """The multi-GPU split of one frame (gravlume_b200.shard.shard_region: a band of whole tile rows
    per rank), each band traced in turn on this GPU into one result set, equals the one-shot frame
    byte for byte."""
    from gravlume_b200.shard import shard_region

    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    with G.TracePipeline(0, G.ReferencePolicy.frame(G.Precision.MIXED)) as pipe:
        one = pipe.trace([sc], [image_camera(0, W, H)])
        banded = TraceResults(W * H, torch.device("cuda", 0))
        for rank in range(world):
            region = shard_region(W, H, world, rank)
            if region is not None:
                pipe.trace([sc], [image_camera(0, W, H, region=region)], banded)
        torch.cuda.synchronize()
    _assert_equal(_bytes(one), _bytes(banded))
