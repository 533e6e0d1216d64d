"""The variational-equation reference gradient of the oracle (oracle/oracle_variational.hpp) on the
CPU: forward-mode sensitivities of the oracle's own binary64 trace, replayed on its accepted steps,
with the implicit-function rule for the event time. Checked against the oracle's central
differences of step-replaying traces (h = 1e-6) on the differentiation workload's rays (a = 0.9,
Q = 0.3, i = 60 deg, r_obs = 50 M, 1024x1024 view)."""

import math

import numpy as np
import pytest

import gravlume_b200 as G
import oracle as O
from gpu_common import oracle_for


@pytest.fixture(scope="module")
def rays():
    a, q, incl, r_obs, n = 0.9, 0.3, math.radians(60.0), 50.0, 1024
    obs = G.Observation.from_oblate(r_obs, incl, 0.0, spin=a, charge=q, chart=G.KerrSchildChart.OUTGOING, width=n,
                                    height=n, vertical_fov=math.radians(30.0), escape_radius=1000.0,
                                    surface=G.EquatorialSurface(G.prograde_isco(a, q), 20.0), horizon_offset=1e-3)
    osc, ev, _ = oracle_for(obs)
    rng = np.random.default_rng(41)
    idx = np.sort(rng.choice(n * n, 256, replace=False))
    states, _, _, status = O.initial_rays(osc, idx % n, idx // n)
    assert (status == 0).all()
    return a, q, ev, np.asarray(states)


def test_variational_gradients_match_central_differences(rays):
    a, q, ev, states = rays
    pol = O.custom_policy(1e-12, 1e-14)
    threads = O.hardware_threads()
    var = O.variational_gradients(1.0, a, q, 1, pol, ev, states, -1.0, threads=threads)
    ind = O.ind_gradients(1.0, a, q, 1, pol, ev, states, -1.0, 1e-6, threads=threads)
    ok = var["ok"] & ind["ok"] & (var["termination"] == ind["termination"])
    # the variational reference differentiates every surface hit and escape; the differences skip
    # the odd ray whose perturbed traces change their step count or class
    assert var["ok"].sum() == np.isin(var["termination"], [O.SURFACE, O.ESCAPE]).sum()
    assert ok.sum() >= var["ok"].sum() - 3
    assert ok.sum() >= 0.8 * len(states)
    np.testing.assert_allclose(var["obs"][ok], ind["obs"][ok], rtol=0, atol=1e-12)
    g1, g2 = var["grad"][ok].reshape(ok.sum(), -1), ind["grad"][ok].reshape(ok.sum(), -1)
    rel = np.abs(g1 - g2).max(axis=1) / np.abs(g1).max(axis=1)
    assert rel.max() <= 1e-6, (np.median(rel), rel.max())
