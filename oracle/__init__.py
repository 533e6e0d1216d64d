"""ctypes bindings for the CPU oracle (test infrastructure only).

The oracle is a binary64 C++ restatement of Gravlume's CPU Dormand-Prince 5(4) reference tracer
(crates/gravlume-reference/src/{integrator,policy,geodesic,events,surface,observation}.rs and the
domain math of crates/gravlume-domain/src/{spacetime,observer,scene,view}.rs). Only the parity
tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may load it; it is the
checker, never the product path.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "_build" / "libgravlume_oracle.so"

# Outcome record layout written by gro_trace_* (one float64 row per ray).
FIELDS = [
    "termination", "failure", "event_kind", "event_candidates", "event_affine", "event_bracket",
    "event_residual", "t", "x", "y", "z", "p_t", "p_x", "p_y", "p_z", "affine_parameter",
    "has_turning_radius", "turning_radius", "azimuth_advance", "travel_time", "polar_side",
    "radial_turnings", "equatorial_crossings", "azimuth_winding", "accepted_steps",
    "rejected_steps", "rhs_evaluations", "minimum_step", "maximum_step", "max_null_residual",
    "max_energy_drift", "max_lz_drift", "max_carter_drift", "has_escape_direction",
    "escape_dx", "escape_dy", "escape_dz", "surface_status", "source_radius", "source_azimuth",
    "frequency_ratio", "emitted_intensity", "observed_intensity",
]
F = {name: i for i, name in enumerate(FIELDS)}

# Termination discriminants (shared with the CUDA path; 1-7 follow the reference's
# TraceTermination, crates/gravlume-render/src/trace.rs:957-967, 8 is the adaptive stepper's
# reject exhaustion).
HORIZON, ESCAPE, SINGULARITY, STEP_EXHAUSTION, NUMERICAL_FAILURE, UNCERTAIN, SURFACE, REJECT_EXHAUSTION = (
    1, 2, 3, 4, 5, 6, 7, 8)


class Policy(ctypes.Structure):
    _fields_ = [
        ("position_rtol", ctypes.c_double), ("position_atol", ctypes.c_double),
        ("momentum_rtol", ctypes.c_double), ("momentum_atol", ctypes.c_double),
        ("initial_step", ctypes.c_double), ("minimum_step", ctypes.c_double),
        ("maximum_step", ctypes.c_double), ("safety", ctypes.c_double),
        ("minimum_factor", ctypes.c_double), ("maximum_factor", ctypes.c_double),
        ("maximum_accepted_steps", ctypes.c_uint64),
        ("maximum_consecutive_rejects", ctypes.c_uint32), ("policy_id", ctypes.c_uint32),
        ("event_affine_tolerance", ctypes.c_double), ("event_tie_tolerance", ctypes.c_double),
        ("event_arming_band", ctypes.c_double), ("singularity_guard", ctypes.c_double),
    ]


class Events(ctypes.Structure):
    _fields_ = [
        ("has_escape", ctypes.c_int32), ("has_surface", ctypes.c_int32),
        ("escape_radius", ctypes.c_double), ("surface_inner", ctypes.c_double),
        ("surface_outer", ctypes.c_double), ("horizon_offset", ctypes.c_double),
        ("intensity_at_six", ctypes.c_double),
    ]


class Scene(ctypes.Structure):
    _fields_ = [
        ("mass", ctypes.c_double), ("spin", ctypes.c_double), ("charge", ctypes.c_double),
        ("chart", ctypes.c_int32), ("pad", ctypes.c_int32),
        ("observer_txyz", ctypes.c_double * 4), ("target_txyz", ctypes.c_double * 4),
        ("up_hint", ctypes.c_double * 3), ("frequency", ctypes.c_double),
        ("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("vertical_fov", ctypes.c_double),
    ]


class ObserverInfo(ctypes.Structure):
    _fields_ = [
        ("event", ctypes.c_double * 4), ("g_tt", ctypes.c_double),
        ("gram_residual", ctypes.c_double), ("orientation", ctypes.c_double),
        ("used_up_fallback", ctypes.c_int32), ("extremality", ctypes.c_int32),
        ("outer_horizon", ctypes.c_double), ("four_velocity", ctypes.c_double * 4),
        ("image_right", ctypes.c_double * 4), ("image_up", ctypes.c_double * 4),
        ("arrival", ctypes.c_double * 4), ("metric_covariant", ctypes.c_double * 16),
        ("tangent_half_fov", ctypes.c_double),
    ]


def _stale() -> bool:
    if not LIB_PATH.exists():
        return True
    t = LIB_PATH.stat().st_mtime
    sources = list(_HERE.glob("*.hpp")) + list(_HERE.glob("*.cpp")) + [_HERE / "Makefile"]
    return any(p.stat().st_mtime > t for p in sources)


def build(force: bool = False) -> Path:
    """Compile the oracle with its Makefile (gcc only; no GPU needed)."""
    if force or _stale():
        subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(str(LIB_PATH))
        dp = ctypes.POINTER(ctypes.c_double)
        L.gro_fields.restype = ctypes.c_int
        L.gro_hardware_threads.restype = ctypes.c_int
        L.gro_policy_preset.argtypes = [ctypes.c_int, ctypes.POINTER(Policy)]
        L.gro_spacetime_info.argtypes = [ctypes.c_double] * 3 + [
            ctypes.c_int, ctypes.POINTER(ctypes.c_int), dp]
        L.gro_oblate_to_cartesian.argtypes = [ctypes.c_double, ctypes.c_int] + [ctypes.c_double] * 3 + [dp]
        L.gro_prograde_isco.argtypes = [ctypes.c_double] * 3
        L.gro_prograde_isco.restype = ctypes.c_double
        L.gro_observer_info.argtypes = [ctypes.POINTER(Scene), ctypes.POINTER(ObserverInfo)]
        L.gro_initial_rays.argtypes = [ctypes.POINTER(Scene), ctypes.c_int64, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
        L.gro_trace_states.argtypes = [ctypes.c_double] * 3 + [
            ctypes.c_int, ctypes.POINTER(Policy), ctypes.POINTER(Events), ctypes.c_int64,
            ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
        L.gro_trace_pixels.argtypes = [ctypes.POINTER(Scene), ctypes.POINTER(Policy),
                                       ctypes.POINTER(Events), ctypes.c_int64, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.gro_surface_observable.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int] + [
            ctypes.c_double] * 3 + [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
        L.gro_invariants.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_void_p,
                                                             ctypes.c_void_p]
        L.gro_hamiltonian_rhs.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_void_p,
                                                                  ctypes.c_void_p]
        assert L.gro_fields() == len(FIELDS)
        _lib = L
    return _lib


def hardware_threads() -> int:
    return int(lib().gro_hardware_threads())


def regular_v1() -> Policy:
    p = Policy()
    lib().gro_policy_preset(0, ctypes.byref(p))
    return p


def strict_v1() -> Policy:
    p = Policy()
    lib().gro_policy_preset(1, ctypes.byref(p))
    return p


def custom_policy(rtol: float, atol: float, **overrides) -> Policy:
    """regular-v1 with both tolerance groups replaced (benchmark workloads use rtol/atol)."""
    p = regular_v1()
    p.position_rtol = p.momentum_rtol = rtol
    p.position_atol = p.momentum_atol = atol
    p.policy_id = 2
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def events(escape_radius=None, surface=None, horizon_offset=0.0, intensity_at_six=1.0) -> Events:
    e = Events()
    e.has_escape = int(escape_radius is not None)
    e.escape_radius = float(escape_radius or 0.0)
    e.has_surface = int(surface is not None)
    if surface is not None:
        e.surface_inner, e.surface_outer = map(float, surface)
    e.horizon_offset = float(horizon_offset)
    e.intensity_at_six = float(intensity_at_six)
    return e


def spacetime_info(mass, spin, charge, chart=0):
    ext = ctypes.c_int()
    rp = ctypes.c_double()
    rc = lib().gro_spacetime_info(mass, spin, charge, chart, ctypes.byref(ext), ctypes.byref(rp))
    if rc != 0:
        raise ValueError("invalid Kerr-Newman parameters")
    return ext.value, rp.value


def oblate_to_cartesian(spin, chart, radius, polar, azimuth):
    out = (ctypes.c_double * 3)()
    lib().gro_oblate_to_cartesian(spin, chart, radius, polar, azimuth, out)
    return list(out)


def prograde_isco(mass, spin, charge) -> float:
    return float(lib().gro_prograde_isco(mass, spin, charge))


def scene(mass=1.0, spin=0.0, charge=0.0, chart=0, observer_txyz=None, observer_oblate=None,
          target=(0.0, 0.0, 0.0, 0.0), up_hint=(0.0, 0.0, 1.0), frequency=1.0, width=1, height=1,
          vertical_fov=0.5) -> Scene:
    s = Scene()
    s.mass, s.spin, s.charge, s.chart = mass, spin, charge, chart
    if observer_txyz is None:
        r, th, ph = observer_oblate
        xyz = oblate_to_cartesian(spin, chart, r, th, ph)
        observer_txyz = (0.0, *xyz)
    s.observer_txyz[:] = list(map(float, observer_txyz))
    s.target_txyz[:] = list(map(float, target))
    s.up_hint[:] = list(map(float, up_hint))
    s.frequency = frequency
    s.width, s.height, s.vertical_fov = width, height, vertical_fov
    return s


def observer_info(sc: Scene) -> ObserverInfo:
    info = ObserverInfo()
    rc = lib().gro_observer_info(ctypes.byref(sc), ctypes.byref(info))
    if rc != 0:
        raise ValueError(f"observer construction failed ({rc})")
    return info


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def initial_rays(sc: Scene, px, py, sx=0.5, sy=0.5):
    px = _c(px, np.uint32)
    n = px.size
    py = _c(py, np.uint32)
    sx = _c(np.broadcast_to(sx, (n,)), np.float64)
    sy = _c(np.broadcast_to(sy, (n,)), np.float64)
    states = np.zeros((n, 8))
    freq = np.zeros(n)
    res = np.zeros(n)
    status = np.zeros(n, np.int32)
    rc = lib().gro_initial_rays(ctypes.byref(sc), n, px.ctypes.data, py.ctypes.data,
                                sx.ctypes.data, sy.ctypes.data, states.ctypes.data,
                                freq.ctypes.data, res.ctypes.data, status.ctypes.data)
    if rc != 0:
        raise ValueError(f"scene construction failed ({rc})")
    return states, freq, res, status


def trace_states(mass, spin, charge, chart, policy, ev, states, direction=1.0, threads=1):
    states = _c(states, np.float64).reshape(-1, 8)
    n = states.shape[0]
    out = np.full((n, len(FIELDS)), np.nan)
    rc = lib().gro_trace_states(mass, spin, charge, chart, ctypes.byref(policy), ctypes.byref(ev),
                                n, states.ctypes.data, direction, threads, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"trace configuration rejected ({rc})")
    return out


def trace_pixels(sc: Scene, policy, ev, px, py, sx=0.5, sy=0.5, threads=1):
    px = _c(px, np.uint32)
    n = px.size
    py = _c(py, np.uint32)
    sx = _c(np.broadcast_to(sx, (n,)), np.float64)
    sy = _c(np.broadcast_to(sy, (n,)), np.float64)
    out = np.full((n, len(FIELDS)), np.nan)
    status = np.zeros(n, np.int32)
    rc = lib().gro_trace_pixels(ctypes.byref(sc), ctypes.byref(policy), ctypes.byref(ev), n,
                                px.ctypes.data, py.ctypes.data, sx.ctypes.data, sy.ctypes.data,
                                threads, out.ctypes.data, status.ctypes.data)
    if rc != 0:
        raise ValueError(f"trace configuration rejected ({rc})")
    return out, status


# Row layout of rk4_pixels (the reference's binary32 GPU RK4 kernel, restated).
RK4_FIELDS = ["termination", "flags", "event_candidates", "steps", "event_residual", "source0", "source1",
              "source2", "travel_time", "null_residual", "energy_drift", "lz_drift", "carter_drift",
              "radial_turnings", "equatorial_crossings", "azimuth_winding"]
RK4 = {name: i for i, name in enumerate(RK4_FIELDS)}


def rk4_pixels(sc: Scene, ev, px, py, sx=0.5, sy=0.5, threads=1):
    """The reference's own GPU algorithm (geodesic_integration.wgsl: binary32 classical RK4 with
    h = clamp(0.1 r, 0.005, 8), at most 2048 steps, Hermite event localization) on image samples;
    a second comparator beside the binary64 oracle. Escape rows hold the unit escape direction in
    source0..2; surface rows hold (radius, azimuth, g)."""
    L = lib()
    L.gro_rk4_pixels.argtypes = [ctypes.POINTER(Scene), ctypes.POINTER(Events), ctypes.c_int64] + [
        ctypes.c_void_p] * 4 + [ctypes.c_int, ctypes.c_void_p]
    px = _c(px, np.uint32)
    n = px.size
    py = _c(py, np.uint32)
    sx = _c(np.broadcast_to(sx, (n,)), np.float64)
    sy = _c(np.broadcast_to(sy, (n,)), np.float64)
    out = np.full((n, len(RK4_FIELDS)), np.nan)
    rc = L.gro_rk4_pixels(ctypes.byref(sc), ctypes.byref(ev), n, px.ctypes.data, py.ctypes.data,
                          sx.ctypes.data, sy.ctypes.data, threads, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"trace configuration rejected ({rc})")
    return out


def surface_observable(mass, spin, charge, chart, inner, outer, state, observer_frequency=1.0,
                       intensity_at_six=1.0):
    """Returns (status, [radius, azimuth, g, emitted, observed]); status 1 = resolved."""
    st = _c(state, np.float64)
    out = np.zeros(5)
    s = lib().gro_surface_observable(mass, spin, charge, chart, inner, outer, intensity_at_six,
                                     st.ctypes.data, observer_frequency, out.ctypes.data)
    return int(s), out


def invariants(mass, spin, charge, chart, state):
    st = _c(state, np.float64)
    out = np.zeros(4)
    rc = lib().gro_invariants(mass, spin, charge, chart, st.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"geometry error {rc}")
    return out


def metric_covariant(mass, spin, charge, chart, txyz):
    """g_{mu nu} at a Cartesian Kerr-Schild event (4x4), or None where the geometry is singular."""
    L = lib()
    L.gro_metric_covariant.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    ev = _c(txyz, np.float64)
    out = np.zeros(16)
    rc = L.gro_metric_covariant(mass, spin, charge, chart, ev.ctypes.data, out.ctypes.data)
    if rc == -1:
        raise ValueError("invalid spacetime parameters")
    return None if rc != 0 else out.reshape(4, 4)


def hamiltonian_rhs(mass, spin, charge, chart, state):
    st = _c(state, np.float64)
    out = np.zeros(8)
    rc = lib().gro_hamiltonian_rhs(mass, spin, charge, chart, st.ctypes.data, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"geometry error {rc}")
    return out


def default_threads() -> int:
    return max(1, int(os.environ.get("GRO_THREADS", "0")) or hardware_threads())


def planck_integral(lo, hi):
    """int_lo^hi x^3 / (e^x - 1) dx by the reference's quadrature (radiation.rs:113-161)."""
    f = lib().gro_planck_integral
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_double, ctypes.c_double]
    return f(lo, hi)


def blackbody_bands(intensity, temperature):
    """Red, green, blue boxcar band intensities of a bolometric intensity at a temperature
    (radiation.rs:13-31); None when not representable."""
    f = lib().gro_blackbody_bands
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    out = np.zeros(3)
    return out if f(intensity, temperature, out.ctypes.data) else None


def surface_radiance(model, intensity_at_six, temperature_at_six, r, g, slab=None):
    """(emitted, observed bolometric, r, g, b) of a surface hit at radius r with frequency ratio g
    (surface.rs:12-72); slab = (optical depth, integrated emission, temperature) or None."""
    f = lib().gro_surface_radiance
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    tau, s, ts = slab if slab is not None else (0.0, 0.0, 0.0)
    out = np.zeros(5)
    ok = f(int(model), intensity_at_six, temperature_at_six, 1 if slab is not None else 0, tau, s, ts, r, g,
           out.ctypes.data)
    return out if ok else None


def surface_footprint(sc: Scene, policy, ev, px, py, sx=0.5, sy=0.5, threads=1):
    """Quarter-pixel surface footprints (footprint.rs:74-150) of pixel samples: (n, 8) rows of
    J (dr/dx, dr/dy, darc/dx, darc/dy; M per pixel), major, minor, determinant, parity (NaN unless
    resolved), and the status per sample (0 no surface, 1 resolved, 2 discontinuity, 3 non-finite)."""
    px = _c(px, np.uint32)
    n = px.size
    py = _c(py, np.uint32)
    sx = _c(np.broadcast_to(sx, (n,)), np.float64)
    sy = _c(np.broadcast_to(sy, (n,)), np.float64)
    out = np.full((n, 8), np.nan)
    status = np.zeros(n, np.int32)
    f = lib().gro_surface_footprint
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    rc = f(ctypes.byref(sc), ctypes.byref(policy), ctypes.byref(ev), n, px.ctypes.data, py.ctypes.data,
           sx.ctypes.data, sy.ctypes.data, threads, out.ctypes.data, status.ctypes.data)
    if rc == -5:
        raise ValueError("surface footprint requires subpixel coordinates in [0.25, 0.75]")
    if rc != 0:
        raise ValueError(f"trace configuration rejected ({rc})")
    return out, status


def footprint_metrics(jacobian):
    """(determinant, squared norm, major, minor) of a 2x2 Jacobian (footprint.rs:203-235), or None
    when it is not finite."""
    f = lib().gro_footprint_metrics
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    j = _c(np.asarray(jacobian, dtype=np.float64).reshape(4), np.float64)
    out = np.zeros(4)
    return out if f(j.ctypes.data, out.ctypes.data) else None


IND_PARAMS = ["p_t", "p_x", "p_y", "p_z", "a", "Q"]
IND_OBS = ["source_radius", "frequency_ratio", "escape_theta", "escape_phi"]


def ind_gradients(mass, spin, charge, chart, policy, ev, states, direction=-1.0, h_rel=1e-6, threads=1):
    """Internal numerical differentiation of traces (the adjoint's check): per ray (termination, ok,
    the 4 observables IND_OBS, then d(observables)/d(param) for IND_PARAMS, param-major), from central
    differences of traces that replay the unperturbed trace's accepted step sizes."""
    states = _c(states, np.float64).reshape(-1, 8)
    n = states.shape[0]
    out = np.zeros((n, 30))
    f = lib().gro_ind_gradients
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int64, ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
    rc = f(mass, spin, charge, chart, ctypes.byref(policy), ctypes.byref(ev), n, states.ctypes.data, direction, h_rel,
           threads, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"spacetime rejected ({rc})")
    return {"termination": out[:, 0].astype(int), "ok": out[:, 1] == 1.0, "obs": out[:, 2:6],
            "grad": out[:, 6:].reshape(n, 6, 4)}


def variational_gradients(mass, spin, charge, chart, policy, ev, states, direction=-1.0, threads=1):
    """Variational-equation reference gradients (forward-mode sensitivities of the oracle's own
    trace, replayed on its accepted steps, with the implicit-function rule for the event time), in
    the layout of ind_gradients: termination, ok, the 4 observables IND_OBS and d(observables)/d(param)
    for IND_PARAMS."""
    states = _c(states, np.float64).reshape(-1, 8)
    n = states.shape[0]
    out = np.zeros((n, 30))
    f = lib().gro_variational_gradients
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_int64, ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
    rc = f(mass, spin, charge, chart, ctypes.byref(policy), ctypes.byref(ev), n, states.ctypes.data, direction,
           threads, out.ctypes.data)
    if rc != 0:
        raise ValueError(f"spacetime rejected ({rc})")
    return {"termination": out[:, 0].astype(int), "ok": out[:, 1] == 1.0, "obs": out[:, 2:6],
            "grad": out[:, 6:].reshape(n, 6, 4)}
