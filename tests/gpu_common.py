"""Shared workload definitions and oracle comparisons for the GPU parity tests."""

from __future__ import annotations

import math

import numpy as np

import gravlume_b200 as G
import oracle as O

F = O.F


def config1_observation(width=256, height=256, spin=0.9, charge=0.3, incl_deg=75.0, r_obs=50.0, chart=1,
                        escape=1000.0, fov_deg=30.0, surface=True, horizon_offset=1e-3):
    """Kerr-Newman a=0.9, Q=0.3 observer at r=50 M, i=75 deg, 30 deg FOV; escape 1000 M, capture at
    r_+ + 1e-3, Keplerian surface from the prograde ISCO to 20 M (the CPU-runnable benchmark case)."""
    surf = G.EquatorialSurface(G.prograde_isco(spin, charge), 20.0) if surface else None
    return G.Observation.from_oblate(r_obs, math.radians(incl_deg), 0.0, spin=spin, charge=charge, chart=chart,
                                     width=width, height=height, vertical_fov=math.radians(fov_deg),
                                     escape_radius=escape, surface=surf, horizon_offset=horizon_offset)


def oracle_for(obs: G.Observation):
    sc = obs.packed
    osc = O.scene(mass=obs.mass, spin=obs.spin, charge=obs.charge, chart=int(obs.chart),
                  observer_txyz=obs.observer_txyz, target=obs.target_txyz, up_hint=obs.up_hint_xyz,
                  width=obs.width, height=obs.height, vertical_fov=obs.vertical_fov)
    surf = (obs.surface.inner_radius, obs.surface.outer_radius) if obs.surface else None
    ev = O.events(escape_radius=obs.escape_radius if obs.escape_radius > 0 else None, surface=surf,
                  horizon_offset=obs.horizon_offset,
                  intensity_at_six=obs.surface.intensity_at_six if obs.surface else 1.0)
    return osc, ev, sc


def seeded_pixels(width, height, n, seed):
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(width * height, size=min(n, width * height), replace=False))
    return idx % width, idx // width


def unit(theta, phi):
    return np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], axis=-1)


# A ray is near-critical when the oracle's own answer moves by more than this between rtol 1e-10
# and rtol 1e-7: its class changes, or its escape direction (rad), hit radius (M) or relative g
# shifts by more than 1e-5, ten times what the looser tolerance moves a well-conditioned ray. On
# the 256x256 frame that is 12 of 65,536 rays: higher-order images that cross the equator two or
# four times before they hit the disk.
NEAR_CRITICAL_SHIFT = 1e-5


def near_critical_band(ref: np.ndarray, loose: np.ndarray) -> np.ndarray:
    """Rays whose class or observables are decided by less than the frame tolerance's truncation:
    `ref` and `loose` are the oracle's rows for the same rays at rtol 1e-10 and rtol 1e-7."""
    t, tl = ref[:, F["termination"]].astype(int), loose[:, F["termination"]].astype(int)
    band = t != tl
    esc = ~band & (t == G.Termination.ESCAPE)
    d0 = np.stack([ref[:, F["escape_dx"]], ref[:, F["escape_dy"]], ref[:, F["escape_dz"]]], axis=1)
    d1 = np.stack([loose[:, F["escape_dx"]], loose[:, F["escape_dy"]], loose[:, F["escape_dz"]]], axis=1)
    ang = np.arccos(np.clip(np.nan_to_num((d0 * d1).sum(1), nan=1.0), -1, 1))
    band |= esc & (ang > NEAR_CRITICAL_SHIFT)
    ref_g = np.where(ref[:, F["frequency_ratio"]] != 0, ref[:, F["frequency_ratio"]], np.nan)
    srf = ~band & (t == G.Termination.EQUATORIAL_SURFACE)
    dr = np.abs(ref[:, F["source_radius"]] - loose[:, F["source_radius"]])
    dg = np.abs(ref[:, F["frequency_ratio"]] - loose[:, F["frequency_ratio"]]) / np.abs(ref_g)
    band |= srf & ((np.nan_to_num(dr) > NEAR_CRITICAL_SHIFT) | (np.nan_to_num(dg) > NEAR_CRITICAL_SHIFT))
    return band


def compare(gpu: dict, sel: np.ndarray, ref: np.ndarray) -> dict:
    """Per-observable max error of GPU rays `sel` against oracle rows `ref` (matching classes only)."""
    gt = gpu["termination"][sel]
    ot = ref[:, F["termination"]].astype(int)
    same = gt == ot
    rep = {"n": int(sel.size), "class_mismatch": int((~same).sum())}
    esc = same & (ot == G.Termination.ESCAPE)
    if esc.any():
        d = np.stack([ref[esc, F["escape_dx"]], ref[esc, F["escape_dy"]], ref[esc, F["escape_dz"]]], axis=1)
        v = unit(gpu["escape_theta"][sel][esc], gpu["escape_phi"][sel][esc])
        rep["escape_direction_rad"] = float(np.max(np.arccos(np.clip(np.sum(d * v, axis=1), -1.0, 1.0))))
    # surface observables exist only for observation traces (oracle surface_status == 1)
    srf = same & (ot == G.Termination.EQUATORIAL_SURFACE) & (ref[:, F["surface_status"]] == 1)
    if srf.any():
        g0 = ref[srf, F["frequency_ratio"]]
        rep["g_rel"] = float(np.max(np.abs(gpu["frequency_ratio"][sel][srf] - g0) / g0))
        rep["hit_radius"] = float(np.max(np.abs(gpu["source_radius"][sel][srf] - ref[srf, F["source_radius"]])))
        dphi = gpu["source_azimuth"][sel][srf] - ref[srf, F["source_azimuth"]]
        rep["source_azimuth"] = float(np.max(np.abs((dphi + np.pi) % (2 * np.pi) - np.pi)))
    if same.any():
        rep["travel_time"] = float(np.max(np.abs(gpu["travel_time"][sel][same] - ref[same, F["travel_time"]])))
        ev = same & np.isfinite(ref[:, F["event_residual"]])
        if ev.any():
            rep["event_residual_gpu_max"] = float(np.nanmax(gpu["event_residual"][sel][ev]))
        for k in ("max_null_residual", "max_lz_drift", "max_carter_drift"):
            rep[k] = float(np.max(np.abs(gpu[k][sel][same] - ref[same, F[k]])))
        if "max_energy_drift" in gpu:
            # E = -p_t is a constant of the stationary metric's Hamiltonian flow in both: zero drift
            rep["max_energy_drift"] = float(np.max(np.abs(gpu["max_energy_drift"][sel][same] -
                                                          ref[same, F["max_energy_drift"]])))
        rep["radial_turnings_mismatch"] = int((gpu["radial_turnings"][sel][same] != ref[same, F["radial_turnings"]]).sum())
        rep["equatorial_crossings_mismatch"] = int(
            (gpu["equatorial_crossings"][sel][same] != ref[same, F["equatorial_crossings"]]).sum())
        if "has_turning_radius" in gpu:
            gh = gpu["has_turning_radius"][sel][same] == 1
            oh = ref[same, F["has_turning_radius"]] == 1
            rep["has_turning_mismatch"] = int((gh != oh).sum())
            both = gh & oh
            if both.any():
                otr = ref[same, F["turning_radius"]][both]
                rep["turning_radius_rel"] = float(np.max(np.abs(gpu["turning_radius"][sel][same][both] - otr) / otr))
    return rep


def pinhole_states(scene, sx, sy):
    """Initial states (t, x, y, z, p_t, p_x, p_y, p_z) of the pinhole rays through image-plane
    points (sx, sy) (tangents of the angles along image-right and image-up), the ray set-up of the
    trace kernels evaluated in numpy for continuous image coordinates."""
    sx = np.atleast_1d(np.asarray(sx, dtype=np.float64))
    sy = np.atleast_1d(np.asarray(sy, dtype=np.float64))
    R = np.array(scene.image_right[:4]); U = np.array(scene.image_up[:4]); A = np.array(scene.arrival[:4])
    u = np.array(scene.four_velocity[:4]); g = np.array(scene.metric_covariant[:16]).reshape(4, 4)
    nrm = 1.0 / np.hypot(1.0, np.hypot(sx, sy))
    sight = (np.outer(sx, R) + np.outer(sy, U) - A) * nrm[:, None]
    pc = scene.frequency * (u - sight)
    p = pc @ g.T
    st = np.zeros((sx.size, 8))
    st[:, :4] = np.array(scene.observer_txyz[:4])
    st[:, 4:] = p
    return st


def near_critical_rays(pipe, spin=0.998, charge=0.05, incl_deg=85.0, r_obs=1000.0, n_dirs=128, n_rays=4096,
                       band=0.05, seed=3, surface=True):
    """The near-critical stress workload: the capture/escape boundary of the observer's image
    (the critical curve) is located along n_dirs radial directions by bisection with the binary64
    kernel at the strict policy, on the scene without its surface; then n_rays rays are drawn with
    impact parameters uniform within +-band M of the curve at seeded directions. Returns the
    observation (with the surface when asked), the states, and each ray's signed distance from the
    curve in M (positive outside)."""
    sky = config1_observation(width=64, height=64, spin=spin, charge=charge, incl_deg=incl_deg, r_obs=r_obs,
                              escape=r_obs, surface=False)
    sc = sky.pack()
    pipe.set_policy(G.ReferencePolicy.strict_v1())
    psi = np.linspace(0.0, 2 * np.pi, n_dirs, endpoint=False)
    lo = np.zeros(n_dirs)               # captured (the image centre looks at the hole)
    hi = np.full(n_dirs, 12.0 / r_obs)  # escapes
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        st = pinhole_states(sc, mid * np.cos(psi), mid * np.sin(psi))
        d = pipe.trace_states(sky, st, direction=-1.0).numpy()
        cap = d["termination"] == G.Termination.HORIZON_CROSSING
        lo = np.where(cap, mid, lo)
        hi = np.where(cap, hi, mid)
    rc = 0.5 * (lo + hi)  # critical radius in the image plane per direction (tangent units)
    rng = np.random.default_rng(seed)
    k = rng.integers(0, n_dirs, n_rays)
    t = rng.uniform(-1.0, 1.0, n_rays)
    # impact parameter b = r_obs * rho for these tiny angles; offsets of +-band M
    rho = rc[k] + t * band / r_obs
    obs = config1_observation(width=64, height=64, spin=spin, charge=charge, incl_deg=incl_deg, r_obs=r_obs,
                              escape=r_obs, surface=surface)
    st = pinhole_states(obs.pack(), rho * np.cos(psi[k]), rho * np.sin(psi[k]))
    return obs, st, (rho - rc[k]) * r_obs
