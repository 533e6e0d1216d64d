"""Post-hit surface transport fused into the trace epilogue (surface.rs:12-72, radiation.rs:13-78,
surface_transport.wgsl): the binary64 kernel's intensities and RGBA16F radiance at every surface
hit of a frame against the oracle's radiation model evaluated at the kernel's own radius and g
(1e-12 relative; binary16 rounding, 2^-11 relative, for the radiance), and the bolometric intensity
against the oracle's full observation trace (its g budget, 1e-8, raised to the fourth power).
"""

import numpy as np
import pytest
import torch

import gravlume_b200 as G
import oracle as O
from gpu_common import F, config1_observation, oracle_for, seeded_pixels

pytestmark = pytest.mark.gpu

CASES = {
    "bolometric": dict(),
    "blackbody_slab": dict(temperature_at_six=9000.0, slab_optical_depth=0.4, slab_emission=0.05,
                           slab_temperature=5000.0),
}


@pytest.fixture(scope="module")
def pipe():
    p = G.TracePipeline(0)
    yield p
    p.close()


def observation(case, n=256):
    obs = config1_observation(width=n, height=n)
    s = obs.surface
    obs.surface = G.EquatorialSurface(s.inner_radius, s.outer_radius, 1.7, **CASES[case])
    return obs


@pytest.mark.parametrize("case", list(CASES))
def test_epilogue_matches_the_radiation_model_at_every_hit(pipe, case):
    obs = observation(case)
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64))
    d = pipe.trace_image(obs).numpy()
    torch.cuda.synchronize()
    hit = d["termination"] == G.Termination.EQUATORIAL_SURFACE
    assert hit.sum() > 1000
    s = obs.surface
    model = 1 if s.temperature_at_six is not None else 0
    slab = (s.slab_optical_depth, s.slab_emission, s.slab_temperature) if s.slab_optical_depth is not None else None
    idx = np.flatnonzero(hit)
    want = np.array([O.surface_radiance(model, 1.7, s.temperature_at_six or 0.0, d["source_radius"][i],
                                        d["frequency_ratio"][i], slab) for i in idx])
    np.testing.assert_allclose(d["emitted_intensity"][idx], want[:, 0], rtol=1e-12)
    np.testing.assert_allclose(d["observed_intensity"][idx], want[:, 1], rtol=1e-12)
    rad = d["radiance"]
    np.testing.assert_allclose(rad[idx, :3], np.minimum(want[:, 2:], 65504.0), rtol=2.0 ** -11, atol=6e-8)
    assert np.all(rad[idx, 3] == 2.0)
    assert np.all(rad[~hit] == 0.0)
    assert np.all(np.isnan(d["observed_intensity"][~hit]))


def test_bolometric_intensity_matches_the_oracle_observation(pipe):
    obs = observation("bolometric")
    osc, ev, _ = oracle_for(obs)
    px, py = seeded_pixels(256, 256, 240, seed=1)
    ref, status = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, px, py, threads=O.hardware_threads())
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.FP64))
    d = pipe.trace_image(obs).numpy()
    torch.cuda.synchronize()
    sel = py * 256 + px
    ok = (ref[:, F["surface_status"]] == 1) & (d["termination"][sel] == G.Termination.EQUATORIAL_SURFACE)
    assert ok.sum() > 20
    for name, field in (("observed_intensity", "observed_intensity"), ("emitted_intensity", "emitted_intensity")):
        rel = np.abs(d[name][sel][ok] - ref[ok, F[field]]) / ref[ok, F[field]]
        assert rel.max() <= 4e-8, (name, rel.max())
