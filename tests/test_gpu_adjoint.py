"""The discrete adjoint on the GPU (glc_forward_ckpt / glc_backward) through the C ABI.

1. Ray lists: the device gradients with respect to the initial momentum, spin and charge equal the
   host-compiled adjoint of the same traces (itself checked against finite differences in
   tests/test_adjoint_host.py) to 1e-8 relative, and do not depend on the checkpoint interval K.
2. Pinhole frames, binary64 and mixed forward passes: the gradients with respect to (a, Q,
   inclination, r_obs), which also flow through the observer tetrad, agree with central differences
   (h = 1e-6) of the binary64 oracle at rtol 1e-12 to 1e-4 relative (the adjoint's precision
   target), both summed over the rays whose termination class is unchanged by the perturbations and
   per ray at the 95th percentile.
"""

import math

import numpy as np
import pytest
import torch

import gravlume_b200 as G
import host_harness as H
import oracle as O
from gpu_common import config1_observation, oracle_for

pytestmark = pytest.mark.gpu

SURF, ESC = G.Termination.EQUATORIAL_SURFACE, G.Termination.ESCAPE


@pytest.fixture(scope="module")
def pipe():
    p = G.TracePipeline(0)
    yield p
    p.close()


def tight(precision=G.Precision.FP64, rtol=1e-12):
    return G.ReferencePolicy.frame(precision, position_rtol=rtol, momentum_rtol=rtol, position_atol=rtol * 1e-2,
                                   momentum_atol=rtol * 1e-2)


def weights(term):
    w = np.zeros((term.size, 4))
    w[term == SURF, 0], w[term == SURF, 1] = 1.0, 10.0
    w[term == ESC, 2], w[term == ESC, 3] = 1.0, 1.0
    return w


def test_ray_list_adjoint_matches_the_host_adjoint_for_every_checkpoint_interval(pipe):
    obs = config1_observation(width=64, height=64)
    osc, ev, sc = oracle_for(obs)
    rng = np.random.default_rng(21)
    states, _, _, status = O.initial_rays(osc, rng.integers(4, 60, 96), rng.integers(4, 60, 96))
    assert (status == 0).all()
    states = np.asarray(states)
    pol = tight()
    base = H.trace_perturbed(sc, pol, states, -1.0)
    w = weights(base[:, 0].astype(int))
    host = H.adjoint_states(sc, pol, states, -1.0, w)
    want_mom = np.stack([-host[:, 6], host[:, 3], host[:, 4], host[:, 5]], axis=1)
    want_par = np.stack([host[:, 7], 2 * 0.3 * host[:, 8]], axis=1)
    pipe.set_policy(pol)
    got = {}
    for K in (1, 4, 64):
        res, tape = pipe.forward_ckpt(obs, 50.0, math.radians(75.0), K=K, states=states)
        g = tape.backward(w)
        torch.cuda.synchronize()
        d = res.numpy()
        np.testing.assert_array_equal(d["termination"], base[:, 0].astype(int))
        got[K] = (g["ray_momentum"].cpu().numpy(), g["ray_params"].cpu().numpy())
        tape.close()
    for K, (mom, par) in got.items():
        scale = np.maximum(np.abs(want_mom).max(axis=1), 1e-300)[:, None]
        err = np.abs(mom - want_mom) / scale
        print("K", K, "momentum max rel", float(err.max()))
        assert err.max() <= 1e-8, K
        perr = np.abs(par[:, :2] - want_par) / np.maximum(np.abs(want_par).max(axis=1), 1e-300)[:, None]
        assert perr.max() <= 1e-8, K
    np.testing.assert_array_equal(got[1][0], got[64][0])


def observation(a, q, incl, r_obs, isco, n):
    return G.Observation.from_oblate(r_obs, incl, 0.0, spin=a, charge=q, chart=G.KerrSchildChart.OUTGOING,
                                     width=n, height=n, vertical_fov=math.radians(30.0), escape_radius=1000.0,
                                     surface=G.EquatorialSurface(isco, 20.0), horizon_offset=1e-3)


def oracle_obs(obs_, px, py):
    osc, ev, _ = oracle_for(obs_)
    ref, status = O.trace_pixels(osc, O.custom_policy(1e-12, 1e-14), ev, px, py, threads=O.hardware_threads())
    assert (status == 0).all()
    F = O.F
    out = np.stack([ref[:, F["source_radius"]], ref[:, F["frequency_ratio"]], np.zeros(len(px)),
                    np.zeros(len(px))], axis=1)
    esc = ref[:, F["termination"]].astype(int) == ESC
    d = np.stack([ref[:, F["escape_dx"]], ref[:, F["escape_dy"]], ref[:, F["escape_dz"]]], axis=1)
    out[esc, 2] = np.arccos(np.clip(d[esc, 2], -1, 1))
    out[esc, 3] = np.arctan2(d[esc, 1], d[esc, 0])
    return ref[:, F["termination"]].astype(int), out


@pytest.mark.parametrize("precision", [G.Precision.FP64, G.Precision.MIXED])
def test_scene_parameter_gradients_match_oracle_central_differences(pipe, precision):
    a, q, incl, r_obs, n = 0.9, 0.3, math.radians(60.0), 50.0, 24
    isco = G.prograde_isco(a, q)
    obs = observation(a, q, incl, r_obs, isco, n)
    pipe.set_policy(tight(G.Precision.FP64, 1e-10) if precision == G.Precision.FP64 else
                    G.ReferencePolicy.frame(G.Precision.MIXED))
    res, tape = pipe.forward_ckpt(obs, r_obs, incl, K=16)
    d = res.numpy()
    term = d["termination"]
    w = weights(term)
    g = tape.backward(w)
    torch.cuda.synchronize()
    per_ray = g["ray_params"].cpu().numpy()
    total = g["params"].cpu().numpy()
    np.testing.assert_allclose(per_ray.sum(axis=0), total, rtol=1e-12, atol=1e-12)
    tape.close()
    idx = np.arange(n * n)
    px, py = idx % n, idx // n
    base_t, base_o = oracle_obs(obs, px, py)
    steps = [1e-6, 1e-6, 1e-6, 1e-6 * r_obs]
    stable = (base_t == term) & np.isin(term, [SURF, ESC])
    fd = np.zeros((n * n, 4))
    params = [a, q, incl, r_obs]
    for k in range(4):
        outs = []
        for sgn in (1, -1):
            p = list(params)
            p[k] += sgn * steps[k]
            t_, o_ = oracle_obs(observation(p[0], p[1], p[2], p[3], isco, n), px, py)
            stable &= t_ == base_t
            outs.append(o_)
        dphi = (outs[0][:, 3] - outs[1][:, 3] + math.pi) % (2 * math.pi) - math.pi
        diff = outs[0] - outs[1]
        diff[:, 3] = dphi
        fd[:, k] = (w * diff).sum(axis=1) / (2 * steps[k])
    # rays whose escape direction sits on the azimuth branch cut or whose observables jump are unstable
    assert stable.sum() >= 0.8 * np.isin(term, [SURF, ESC]).sum()
    adj_sum = per_ray[stable].sum(axis=0)
    fd_sum = fd[stable].sum(axis=0)
    rel = np.abs(adj_sum - fd_sum) / np.maximum(np.abs(fd_sum), 1e-12)
    scale = np.maximum(np.abs(fd[stable]).max(axis=1), 1e-12)
    per_rel = np.abs(per_ray[stable] - fd[stable]).max(axis=1) / scale
    print(precision.name, "adjoint", adj_sum, "fd", fd_sum, "rel", rel, "per-ray median", np.median(per_rel),
          "p95", np.quantile(per_rel, 0.95))
    assert np.all(rel <= 1e-4), rel
    assert np.quantile(per_rel, 0.95) <= 1e-4


def test_reused_tape_gives_the_fresh_tapes_gradients(pipe):
    """glc_forward_ckpt_into: a tape reused across an optimization step (the scene's spin changed in
    between, then changed back) gives bit-identical results and per-ray gradients to fresh tapes, and
    does not grow its memory when the request fits."""
    a, q, incl, r_obs, n = 0.9, 0.3, math.radians(60.0), 50.0, 32
    isco = G.prograde_isco(a, q)
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED))
    obs0, obs1 = observation(a, q, incl, r_obs, isco, n), observation(a - 0.01, q, incl, r_obs, isco, n)

    def grads(tape, res):
        w = weights(res.numpy()["termination"])
        g = tape.backward(w)
        torch.cuda.synchronize()
        return res.numpy(), g["ray_momentum"].cpu().numpy(), g["params"].cpu().numpy()

    fresh = []
    for o in (obs0, obs1):
        res, tape = pipe.forward_ckpt(o, r_obs, incl, K=16)
        fresh.append(grads(tape, res))
        tape.close()
    res, tape = pipe.forward_ckpt(obs0, r_obs, incl, K=16)
    grads(tape, res)
    before = tape.info()["bytes"]
    for o, want in ((obs1, fresh[1]), (obs0, fresh[0])):
        got = grads(tape, tape.forward_again(o))
        np.testing.assert_array_equal(got[0]["termination"], want[0]["termination"])
        np.testing.assert_array_equal(got[0]["source_radius"], want[0]["source_radius"])
        np.testing.assert_array_equal(got[1], want[1])
        # the scene gradient is summed over rays by atomics, in no fixed order
        np.testing.assert_allclose(got[2], want[2], rtol=1e-13)
    assert tape.info()["bytes"] == before
    tape.close()


@pytest.mark.parametrize("precision", [G.Precision.FP64, G.Precision.MIXED])
def test_ray_gradients_match_the_oracles_internal_numerical_differentiation(pipe, precision):
    """The differentiation workload's rays (a = 0.9, Q = 0.3, i = 60 deg, r = 50 M; 1024 seeded pixels
    of the 1024x1024 frame): the device adjoint's per-ray gradients with respect to (p_t, p_x, p_y,
    p_z) and to a and Q in the dynamics, against the oracle's internal numerical differentiation at
    rtol 1e-12 (central differences of traces replaying the unperturbed trace's steps). The binary64
    forward at rtol 1e-12 agrees to 1e-6 of each gradient's largest component; the MIXED forward at
    the frame tolerance carries its rtol 7e-7 truncation, and the adjoint's precision target, 1e-4,
    is asked of 95 % of its rays."""
    a, q, incl, r_obs, n = 0.9, 0.3, math.radians(60.0), 50.0, 1024
    isco = G.prograde_isco(a, q)
    obs = observation(a, q, incl, r_obs, isco, n)
    osc, ev, _ = oracle_for(obs)
    rng = np.random.default_rng(40)
    idx = np.sort(rng.choice(n * n, 1024, replace=False))
    states, _, _, status = O.initial_rays(osc, idx % n, idx // n)
    assert (status == 0).all()
    states = np.asarray(states)
    ind = O.ind_gradients(1.0, a, q, 1, O.custom_policy(1e-12, 1e-14), ev, states, -1.0, 1e-6,
                          threads=O.hardware_threads())
    keep = ind["ok"]
    assert keep.mean() >= 0.95
    w = weights(ind["termination"])
    want = np.einsum("npk,nk->np", ind["grad"], w)
    pipe.set_policy(tight() if precision == G.Precision.FP64 else G.ReferencePolicy.frame(G.Precision.MIXED))
    res, tape = pipe.forward_ckpt(obs, r_obs, incl, K=64, states=states)
    d = res.numpy()
    g = tape.backward(w)
    torch.cuda.synchronize()
    got = np.concatenate([g["ray_momentum"].cpu().numpy(), g["ray_params"].cpu().numpy()[:, :2]], axis=1)
    tape.close()
    keep &= d["termination"] == ind["termination"]
    rel = np.abs(got[keep] - want[keep]).max(axis=1) / np.abs(want[keep]).max(axis=1)
    print(precision.name, "rays", int(keep.sum()), "median", float(np.median(rel)), "p95",
          float(np.quantile(rel, 0.95)), "max", float(rel.max()))
    if precision == G.Precision.FP64:
        assert rel.max() <= 1e-6
    else:
        assert np.quantile(rel, 0.95) <= 1e-4


def test_failed_forward_into_a_tape_blocks_its_backward(pipe):
    """A forward pass into a reused tape that the library rejects (here a view of another size than
    the tape's camera) leaves the tape unusable for glc_backward until a forward pass succeeds."""
    a, q, incl, r_obs, n = 0.9, 0.3, math.radians(60.0), 50.0, 16
    isco = G.prograde_isco(a, q)
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED))
    obs = observation(a, q, incl, r_obs, isco, n)
    res, tape = pipe.forward_ckpt(obs, r_obs, incl, K=16)
    w = weights(res.numpy()["termination"])
    tape.backward(w)
    with pytest.raises(G.GlcError, match="size"):
        tape.forward_again(observation(a, q, incl, r_obs, isco, n + 8))
    with pytest.raises(G.GlcError, match="failed"):
        tape.backward(w)
    res = tape.forward_again(obs)
    g = tape.backward(w)
    torch.cuda.synchronize()
    assert np.isfinite(g["ray_momentum"].cpu().numpy()).all()
    tape.close()


@pytest.fixture(scope="module")
def differentiation_subsample():
    """The differentiation workload's seeded 4096-ray subsample (a = 0.9, Q = 0.3, i = 60 deg,
    r_obs = 50 M, 1024x1024 view) with both binary64 references at rtol 1e-12: the oracle's
    variational-equation gradient and its central differences (h = 1e-6) of step-replaying traces."""
    a, q, incl, r_obs, n = 0.9, 0.3, math.radians(60.0), 50.0, 1024
    isco = G.prograde_isco(a, q)
    obs = observation(a, q, incl, r_obs, isco, n)
    osc, ev, _ = oracle_for(obs)
    rng = np.random.default_rng(4096)
    idx = np.sort(rng.choice(n * n, 4096, replace=False))
    states, _, _, status = O.initial_rays(osc, idx % n, idx // n)
    assert (status == 0).all()
    states = np.asarray(states)
    pol = O.custom_policy(1e-12, 1e-14)
    threads = O.hardware_threads()
    var = O.variational_gradients(1.0, a, q, 1, pol, ev, states, -1.0, threads=threads)
    ind = O.ind_gradients(1.0, a, q, 1, pol, ev, states, -1.0, 1e-6, threads=threads)
    return obs, r_obs, incl, states, var, ind


@pytest.mark.parametrize("precision", [G.Precision.FP64, G.Precision.MIXED])
@pytest.mark.parametrize("K", [16, 64, 256])
def test_ray_gradients_match_the_variational_reference(pipe, differentiation_subsample, precision, K):
    """Per-ray gradients of the weighted observables with respect to (p_t, p_x, p_y, p_z, a, Q) on
    every differentiated ray of the 4096-ray subsample: the binary64 forward at rtol 1e-12 within
    1e-6, and the MIXED forward at the frame tolerance within the adjoint's target 1e-4, of each
    ray's largest gradient component, against the variational reference; the central differences
    agree with the variational reference to 1e-6 on the same rays."""
    obs, r_obs, incl, states, var, ind = differentiation_subsample
    w = weights(var["termination"])
    want = np.einsum("npk,nk->np", var["grad"], w)
    both = var["ok"] & ind["ok"] & (var["termination"] == ind["termination"])
    fd = np.einsum("npk,nk->np", ind["grad"], w)
    fd_rel = np.abs(fd[both] - want[both]).max(axis=1) / np.abs(want[both]).max(axis=1)
    assert fd_rel.max() <= 1e-6, fd_rel.max()
    pipe.set_policy(tight() if precision == G.Precision.FP64 else G.ReferencePolicy.frame(G.Precision.MIXED))
    res, tape = pipe.forward_ckpt(obs, r_obs, incl, K=K, states=states)
    d = res.numpy()
    g = tape.backward(w)
    torch.cuda.synchronize()
    got = np.concatenate([g["ray_momentum"].cpu().numpy(), g["ray_params"].cpu().numpy()[:, :2]], axis=1)
    tape.close()
    keep = var["ok"] & (d["termination"] == var["termination"])
    assert keep.sum() >= 0.95 * var["ok"].sum()
    rel = np.abs(got[keep] - want[keep]).max(axis=1) / np.abs(want[keep]).max(axis=1)
    print(precision.name, "K", K, "rays", int(keep.sum()), "median", float(np.median(rel)), "max", float(rel.max()))
    assert rel.max() <= (1e-6 if precision == G.Precision.FP64 else 1e-4), rel.max()
