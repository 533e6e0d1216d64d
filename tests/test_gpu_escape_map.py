"""Escape-direction map (crates/gravlume-render/src/shaders/geodesic_acceleration.wgsl:330-586): a
node pass traces every 4th pixel of each axis and stores each node in the reference's packed
format (2-bit tag, 15 + 15-bit octahedral direction); stable 8x8 tiles of surface-free scenes are
reconstructed by bilinear interpolation of their 3x3 node stencil.

Checked against full binary64 integration of the same frame: reconstructed pixels escape, within
the reference's 3.82e-4 rad direction budget; node pixels and every traced pixel are unchanged;
scenes with a surface are never reconstructed.
"""

import numpy as np
import pytest
import torch

import gravlume_b200 as G
from gravlume_b200 import _native as N
from gpu_common import config1_observation, unit

pytestmark = pytest.mark.gpu

RECONSTRUCTED = 32  # bit 25 of code.x, bit 5 of the decoded flags
BUDGET = 3.82e-4


@pytest.fixture(scope="module")
def pipe():
    p = G.TracePipeline(0)
    yield p
    p.close()


def frame(pipe, scene, cam, slots, escape_map):
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64, position_rtol=1e-8, momentum_rtol=1e-8,
                                            position_atol=1e-10, momentum_atol=1e-10, maximum_step=1000.0,
                                            escape_map=int(escape_map)))
    res = G.TraceResults(slots, "cuda")
    pipe.trace([scene], [cam], res)
    torch.cuda.synchronize()
    return res.numpy()


def check(on, off, w, h, min_fraction):
    rec = (on["flags"] & RECONSTRUCTED) != 0
    esc = off["termination"] == G.Termination.ESCAPE
    assert np.all(esc[rec]), "a reconstructed pixel does not escape under full integration"
    ang = np.arccos(np.clip(np.sum(unit(on["escape_theta"][rec], on["escape_phi"][rec]) *
                                   unit(off["escape_theta"][rec], off["escape_phi"][rec]), axis=1), -1, 1))
    frac = rec.sum() / max(esc.sum(), 1)
    print("reconstructed", int(rec.sum()), "of", int(esc.sum()), "escapes;", "max angle", float(ang.max()),
          "median", float(np.median(ang)))
    assert ang.max() <= BUDGET
    assert frac >= min_fraction
    # node pixels (every 4th of each axis) are traced in full by the node pass
    node = np.zeros((h, w), bool)
    node[::4, ::4] = True
    node = node.ravel()
    np.testing.assert_array_equal(on["termination"][node], off["termination"][node])
    np.testing.assert_array_equal(on["accepted_steps"][node], off["accepted_steps"][node])
    traced = ~rec
    np.testing.assert_array_equal(on["termination"][traced], off["termination"][traced])
    np.testing.assert_allclose(on["travel_time"][traced], off["travel_time"][traced], rtol=1e-9, atol=1e-9,
                               equal_nan=True)


def test_pinhole_sky_reconstruction_stays_within_the_direction_budget(pipe):
    w = h = 768
    obs = config1_observation(width=w, height=h, surface=False)
    sc = obs.pack()
    cam = G.image_camera(0, w, h)
    check(frame(pipe, sc, cam, w * h, True), frame(pipe, sc, cam, w * h, False), w, h, 0.3)


def test_equirect_escape_map_reconstruction(pipe):
    w, h = 2048, 1024
    sky = config1_observation(width=64, height=64, r_obs=15.0, incl_deg=60.0, surface=False)
    sc = sky.pack()
    cam = G.image_camera(0, w, h, kind=N.CAMERA_EQUIRECT)
    check(frame(pipe, sc, cam, w * h, True), frame(pipe, sc, cam, w * h, False), w, h, 0.3)


def test_scenes_with_a_surface_are_traced_in_full(pipe):
    obs = config1_observation(width=256, height=256)
    sc = obs.pack()
    on = frame(pipe, sc, G.image_camera(0, 256, 256), 256 * 256, True)
    assert not np.any(on["flags"] & RECONSTRUCTED)
