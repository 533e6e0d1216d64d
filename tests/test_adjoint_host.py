"""The discrete adjoint's reverse sweeps (gravlume_b200/csrc/glc_adjoint.cuh, compiled for the host
by the test harness) against central finite differences of the same tracer.

For each ray, the gradient of L = w . (source radius, g, escape theta, escape phi) with respect to the
initial position and momentum, E, the spin a and Q^2 (in the dynamics) is compared with central
differences of L over whole traces at the binary64 policy rtol 1e-12, step 1e-6 (relative to the
variable's scale). Tolerance: 1e-4 relative to the gradient's largest component, the precision
target of the adjoint. The finite differences include the controller's response to the perturbation,
which is O(tolerance / step) = 1e-6 here.
"""

import numpy as np
import pytest

import gravlume_b200 as G
import host_harness as H
import oracle as O
from gpu_common import config1_observation, oracle_for

REL = 1e-4


@pytest.fixture(scope="module")
def rays():
    obs = config1_observation(width=64, height=64)
    osc, ev, sc = oracle_for(obs)
    rng = np.random.default_rng(21)
    px, py = rng.integers(8, 56, 40), rng.integers(8, 56, 40)
    states, _, _, status = O.initial_rays(osc, px, py)
    assert (status == 0).all()
    pol = G.ReferencePolicy.frame(G.Precision.FP64, position_rtol=1e-12, momentum_rtol=1e-12,
                                  position_atol=1e-14, momentum_atol=1e-14)
    base = H.trace_perturbed(sc, pol, states, -1.0)
    keep = np.isin(base[:, 0], [G.Termination.EQUATORIAL_SURFACE, G.Termination.ESCAPE])
    return sc, pol, np.asarray(states)[keep][:12], base[keep][:12]


def weights(term):
    w = np.zeros((term.size, 4))
    srf = term == G.Termination.EQUATORIAL_SURFACE
    w[srf, 0], w[srf, 1] = 1.0, 10.0
    w[~srf, 2], w[~srf, 3] = 1.0, 1.0
    return w


def loss(obs, w):
    v = np.nan_to_num(obs[:, 1:5]) * w
    return v.sum(axis=1)


def test_adjoint_matches_finite_differences_of_the_trace(rays):
    sc, pol, states, base = rays
    assert len(states) >= 6
    term = base[:, 0].astype(int)
    assert (term == G.Termination.EQUATORIAL_SURFACE).any() and (term == G.Termination.ESCAPE).any()
    w = weights(term)
    adj = H.adjoint_states(sc, pol, states, -1.0, w)
    assert np.all(adj[:, 10] == 1.0)
    fd = np.zeros((len(states), 9))
    # state components: (x, y, z) = st8[1..3], (p_x, p_y, p_z) = st8[5..7], E = -st8[4]
    cols = [1, 2, 3, 5, 6, 7, 4]
    for k, col in enumerate(cols):
        eps = 1e-6 * max(1.0, float(np.max(np.abs(states[:, col]))))
        sp, sm = states.copy(), states.copy()
        sp[:, col] += eps
        sm[:, col] -= eps
        lp = loss(H.trace_perturbed(sc, pol, sp, -1.0), w)
        lm = loss(H.trace_perturbed(sc, pol, sm, -1.0), w)
        fd[:, k] = (lp - lm) / (2 * eps)
    fd[:, 6] *= -1.0  # dL/dE = -dL/dp_t
    for k, (da, dq) in ((7, (1e-6, 0.0)), (8, (0.0, 1e-6))):
        lp = loss(H.trace_perturbed(sc, pol, states, -1.0, da, dq), w)
        lm = loss(H.trace_perturbed(sc, pol, states, -1.0, -da, -dq), w)
        fd[:, k] = (lp - lm) / (2 * (da + dq))
    for i in range(len(states)):
        scale = np.max(np.abs(fd[i]))
        err = np.max(np.abs(adj[i, :9] - fd[i])) / scale
        assert err <= REL, (i, int(term[i]), err, adj[i, :9], fd[i])


def test_hamiltonian_stage_vjp_equals_the_jacobian_transpose():
    """The sweeps' 4-channel stage VJP (F = J grad H, so J_y^T kbar = Hess(H) J^T kbar) against the
    9-channel Jacobian transpose at seeded states along the frame's rays and random cotangents."""
    obs = config1_observation(width=64, height=64)
    osc, ev, sc = oracle_for(obs)
    rng = np.random.default_rng(4)
    px, py = rng.integers(0, 64, 64), rng.integers(0, 64, 64)
    states, _, _, status = O.initial_rays(osc, px, py)
    st = np.asarray(states)
    # points along the rays, from the observer inwards (first-order moves keep them off the horizon)
    t = rng.uniform(0.0, 40.0, (64, 1))
    y = np.concatenate([st[:, 1:4] + t * st[:, 5:8] / np.linalg.norm(st[:, 5:8], axis=1, keepdims=True),
                        st[:, 5:8]], axis=1)
    kbar = rng.normal(size=(64, 6))
    out = H.rhs_vjp_pair(sc, y, -st[:, 4], kbar)
    a, b = out[:, :9], out[:, 9:]
    scale = np.max(np.abs(b), axis=1, keepdims=True)
    assert np.all(np.isfinite(a))
    assert np.all(np.abs(a - b) <= 1e-12 * scale)


def test_adjoint_matches_the_oracles_internal_numerical_differentiation(rays):
    """The sweeps' gradient with respect to (p_t, p_x, p_y, p_z, a, Q) against the oracle's internal
    numerical differentiation: central differences (h = 1e-6) of oracle traces at rtol 1e-12 that
    replay the unperturbed trace's accepted steps, i.e. the tangent of the oracle's own discrete map.
    The two maps take different step sequences at the same tolerance, so they agree to the
    integration accuracy; 1e-6 of the gradient's largest component is asked."""
    sc, pol, states, base = rays
    obs = config1_observation(width=64, height=64)
    osc, ev, _ = oracle_for(obs)
    ind = O.ind_gradients(1.0, 0.9, 0.3, 1, O.custom_policy(1e-12, 1e-14), ev, states, -1.0, 1e-6,
                          threads=O.default_threads())
    assert ind["ok"].all()
    term = ind["termination"]
    w = weights(term)
    host = H.adjoint_states(sc, pol, states, -1.0, w)
    assert (host[:, 10] == 1.0).all()
    adj = np.stack([-host[:, 6], host[:, 3], host[:, 4], host[:, 5], host[:, 7], 2 * 0.3 * host[:, 8]], axis=1)
    want = np.einsum("npk,nk->np", ind["grad"], w)
    rel = np.abs(adj - want).max(axis=1) / np.abs(want).max(axis=1)
    assert rel.max() <= 1e-6, rel.max()
