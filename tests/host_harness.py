"""Builds and loads tests/native/host_trace.cpp: the device tracer's per-ray logic compiled for the
host (test infrastructure; the product path is the CUDA kernel)."""

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "native" / "host_trace.cpp"
OUT = ROOT / "tests" / "native" / "_build" / "libhost_trace.so"
DEPS = [SRC] + sorted((ROOT / "gravlume_b200" / "csrc").glob("*.cuh")) + [ROOT / "include" / "glc.h"]

FIELDS = ["termination", "failure", "candidates", "flags", "accepted_steps", "rejected_steps",
          "radial_turnings", "equatorial_crossings", "azimuth_winding", "escape_theta", "escape_phi",
          "source_radius", "source_azimuth", "frequency_ratio", "travel_time", "event_residual",
          "affine_parameter", "max_null_residual", "max_lz_drift", "max_carter_drift", "turning_radius",
          "azimuth_advance", "x", "y", "z", "p_x", "p_y", "p_z", "f64_steps"]

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not OUT.exists() or any(d.stat().st_mtime > OUT.stat().st_mtime for d in DEPS):
            OUT.parent.mkdir(parents=True, exist_ok=True)
            subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-x", "c++", str(SRC), "-o", str(OUT)],
                           check=True)
        L = ctypes.CDLL(str(OUT))
        L.host_trace_states.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                        ctypes.c_double, ctypes.c_void_p]
        L.host_adjoint_states.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                          ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        L.host_trace_perturbed.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
        assert L.host_trace_fields() == len(FIELDS)
        _lib = L
    return _lib


def trace_states(scene, policy, states, direction):
    st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
    out = np.zeros((st.shape[0], len(FIELDS)))
    rc = lib().host_trace_states(ctypes.byref(scene), ctypes.byref(policy), st.shape[0], st.ctypes.data,
                                 direction, out.ctypes.data)
    assert rc == 0
    d = {k: out[:, i] for i, k in enumerate(FIELDS)}
    d["termination"] = d["termination"].astype(int)
    return d


def trace_split(scene, policy, states, direction):
    """MIXED as two kernels: the binary32 bulk stepper until its hand-off, the 128-byte hand-off
    record, then the binary64 completion (the device kernels' per-ray logic, compiled for the host)."""
    st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
    out = np.zeros((st.shape[0], len(FIELDS)))
    f = lib().host_trace_split
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_double,
                  ctypes.c_void_p]
    assert f(ctypes.byref(scene), ctypes.byref(policy), st.shape[0], st.ctypes.data, direction,
             out.ctypes.data) == 0
    d = {k: out[:, i] for i, k in enumerate(FIELDS)}
    d["termination"] = d["termination"].astype(int)
    return d


def adjoint_states(scene, policy, states, direction, dl_dobs):
    """Per ray: dL/d(x, y, z, p_x, p_y, p_z) at the initial state, dL/dE, dL/da, dL/dQ^2,
    termination, ok flag, accepted steps (the device adjoint's sweeps, compiled for the host)."""
    st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
    w = np.ascontiguousarray(dl_dobs, dtype=np.float64).reshape(-1, 4)
    out = np.zeros((st.shape[0], 12))
    rc = lib().host_adjoint_states(ctypes.byref(scene), ctypes.byref(policy), st.shape[0], st.ctypes.data,
                                   direction, w.ctypes.data, out.ctypes.data)
    assert rc == 0
    return out


def trace_perturbed(scene, policy, states, direction, da=0.0, dq2=0.0):
    """Termination, source radius, g, escape theta, escape phi under spin/charge^2 shifted in the dynamics."""
    st = np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)
    out = np.zeros((st.shape[0], 5))
    rc = lib().host_trace_perturbed(ctypes.byref(scene), ctypes.byref(policy), st.shape[0], st.ctypes.data,
                                    direction, da, dq2, out.ctypes.data)
    assert rc == 0
    return out


def blackbody_bands(intensity, temperature):
    f = lib().host_blackbody_bands
    f.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    out = np.zeros(3)
    return out if f(intensity, temperature, out.ctypes.data) else None


def surface_radiance(model, i6, t6, r, g, slab=None):
    f = lib().host_surface_radiance
    f.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p]
    tau, s, ts = slab if slab is not None else (0.0, 0.0, 0.0)
    out = np.zeros(5)
    return out if f(int(model), i6, t6, 1 if slab is not None else 0, tau, s, ts, r, g, out.ctypes.data) else None


def rhs_vjp_pair(scene, y, E, kbar):
    """(n, 18): ybar and dL/d(E, a, Q^2) from the 4-channel Hamiltonian stage VJP, then from the
    9-channel Jacobian."""
    f = lib().host_rhs_vjp_pair
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    y = np.ascontiguousarray(y, dtype=np.float64).reshape(-1, 6)
    E = np.ascontiguousarray(E, dtype=np.float64).reshape(-1)
    kb = np.ascontiguousarray(kbar, dtype=np.float64).reshape(-1, 6)
    out = np.zeros((y.shape[0], 18))
    assert f(ctypes.byref(scene), y.shape[0], y.ctypes.data, E.ctypes.data, kb.ctypes.data, out.ctypes.data) == 0
    return out
