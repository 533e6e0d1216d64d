"""The end-to-end host-buffer call (glc_trace_host) against the device-buffer trace of the same job.

A job large enough to be traced in bands, with its results copied back band by band on a second
stream while later bands are traced, holds a 2048x1024 pinhole frame (four row bands of 2^19
rays) and a ray list behind it in the result slots. Its every result array must equal the device
trace's byte for byte, in binary32 and binary64 (the same kernel traces every ray either way). A
MIXED frame is compared the same way: its bands start on whole tile rows, so each warp holds the
same rays as in the one-launch trace, and its warp-wide binary64 decisions are the same. The
persistent kernel, whose launches are not banded, goes through the one-launch path and must match
as well.
"""

import math

import numpy as np
import pytest
import torch

import gravlume_b200 as G
from gpu_common import config1_observation, pinhole_states

pytestmark = pytest.mark.gpu

W, H, NL = 2048, 1024, 3000


@pytest.fixture(scope="module")
def job():
    obs = config1_observation(width=W, height=H)
    sc = obs.pack()
    rng = np.random.default_rng(8)
    t = math.tan(math.radians(15.0))
    states = np.ascontiguousarray(pinhole_states(sc, rng.uniform(-2 * t, 2 * t, NL), rng.uniform(-t, t, NL)))
    return sc, states


def cameras(states_ptr):
    return [G.image_camera(0, W, H), G.raylist_camera(0, states_ptr, NL, -1.0, offset=W * H)]


@pytest.fixture(scope="module")
def pipe():
    p = G.TracePipeline(0)
    yield p
    p.close()


def compare(pipe, sc, states, image_only=False):
    dev_states = torch.as_tensor(states).cuda()
    dev_cams = cameras(dev_states.data_ptr())
    host_cams = cameras(states.ctypes.data)
    if image_only:
        dev_cams, host_cams = dev_cams[:1], host_cams[:1]
    dev = pipe.trace([sc], dev_cams)
    torch.cuda.synchronize()
    host = pipe.trace_host([sc], host_cams)
    n = W * H + (0 if image_only else NL)
    for name, buf in dev.buffers.items():
        a = buf.cpu().numpy()[:n]
        b = host.buffers[name].numpy()[:n]
        assert np.array_equal(a, b), name
    d = host.numpy()
    assert (d["termination"][:n] > 0).all()
    return d


@pytest.mark.parametrize("precision", [G.Precision.FP32, G.Precision.FP64])
def test_banded_host_trace_equals_the_device_trace(pipe, job, precision):
    sc, states = job
    pipe.set_policy(G.ReferencePolicy.frame(precision))
    before = pipe.stats().kernel_launches
    compare(pipe, sc, states)
    # one device trace, then five bands (four row bands of the frame, one of the ray list)
    assert pipe.stats().kernel_launches - before == 1 + 5


def test_banded_mixed_frame_equals_the_device_trace(pipe, job):
    sc, states = job
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED))
    compare(pipe, sc, states, image_only=True)


def test_persistent_policy_takes_the_one_launch_path(pipe, job):
    sc, states = job
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP32, persistent=2))
    compare(pipe, sc, states)
