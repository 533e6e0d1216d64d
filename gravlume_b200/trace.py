"""Python host API over the C ABI, in the reference's terms.

The names mirror the reference's trace boundary so that callers and tests read the same way:
``Observation`` (crates/gravlume-domain/src/scene.rs:183-271) bundles the physical scene,
stationary observer and perspective view; ``ReferencePolicy`` (crates/gravlume-reference/src/
policy.rs:26-66) the step policy; ``TracePipeline`` (crates/gravlume-render/src/trace.rs:320-327,
701-710) the device pipeline; ``Termination`` (crates/gravlume-reference/src/outcome.rs:150-158 /
crates/gravlume-render/src/trace.rs:957-967) the discrete outcome. Every trace runs the sm_100a
kernels in libglc.so; there is no CPU path.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from enum import IntEnum
from typing import Iterable, Sequence

import numpy as np

from . import _native as N


class KerrSchildChart(IntEnum):
    INGOING = 0
    OUTGOING = 1


class Precision(IntEnum):
    FP32 = 0
    MIXED = 1
    FP64 = 2


class Termination(IntEnum):
    HORIZON_CROSSING = 1
    ESCAPE = 2
    SINGULARITY_GUARD = 3
    STEP_EXHAUSTION = 4
    NUMERICAL_FAILURE = 5
    UNCERTAIN = 6
    EQUATORIAL_SURFACE = 7
    REJECT_EXHAUSTION = 8


class FootprintStatus(IntEnum):
    """Per-pixel outcome of glc_surface_footprint (footprint.rs:12-16, 258-268)."""
    NO_SURFACE = 0
    RESOLVED = 1
    DISCONTINUITY = 2
    NON_FINITE = 3


FOOTPRINT_QUARTER_PIXEL = 0
FOOTPRINT_TANGENT = 1


def footprint_fields(fp) -> dict:
    """Split the (slots, 8) footprint array of TracePipeline.surface_footprint (a tensor or a numpy
    array) into numpy fields: jacobian (slots, 2, 2; rows radius and local arc, columns screen x and
    y), singular_values (slots, 2), determinant, status and parity."""
    a = fp.cpu().numpy() if hasattr(fp, "cpu") else np.asarray(fp)
    a = np.ascontiguousarray(a, dtype=np.float64)
    tail = a[:, 7].copy().view(np.int32).reshape(-1, 2)
    return {"jacobian": a[:, :4].reshape(-1, 2, 2), "singular_values": a[:, 4:6], "determinant": a[:, 6],
            "status": tail[:, 0].copy(), "parity": tail[:, 1].copy()}


def oblate_to_cartesian(spin: float, chart: int, radius: float, polar: float, azimuth: float):
    """KerrNewmanSpacetime::oblate_to_cartesian (crates/gravlume-domain/src/spacetime.rs:245-254)."""
    st, ct = math.sin(polar), math.cos(polar)
    sp, cp = math.sin(azimuth), math.cos(azimuth)
    cs = (1.0 if int(chart) == 0 else -1.0) * spin
    return [(cs * -sp + radius * cp) * st, (cs * cp + radius * sp) * st, radius * ct]


def prograde_isco(spin: float, charge: float = 0.0) -> float:
    out = ctypes.c_double()
    N.check(N.lib().glc_prograde_isco(spin, charge, ctypes.byref(out)), "glc_prograde_isco")
    return out.value


@dataclass
class EquatorialSurface:
    """Inclusive radial interval of the Keplerian emitter (emission.rs:30-41): inverse-cube
    bolometric intensity I(6 M), or inverse-cube blackbody with temperature T(6 M) when
    `temperature_at_six` is given; an optional homogeneous scalar slab in front of it (optical depth,
    integrated bolometric emission, and the slab temperature for the blackbody band split)."""
    inner_radius: float
    outer_radius: float
    intensity_at_six: float = 1.0
    temperature_at_six: float | None = None
    slab_optical_depth: float | None = None
    slab_emission: float = 0.0
    slab_temperature: float = 0.0


@dataclass
class Observation:
    """A validated physical scene + stationary observer + perspective view + events."""
    mass: float = 1.0
    spin: float = 0.0
    charge: float = 0.0
    chart: int = KerrSchildChart.OUTGOING
    observer_txyz: Sequence[float] = (0.0, 50.0, 0.0, 0.0)
    target_txyz: Sequence[float] = (0.0, 0.0, 0.0, 0.0)
    up_hint_xyz: Sequence[float] = (0.0, 0.0, 1.0)
    measured_frequency: float = 1.0
    width: int = 256
    height: int = 256
    vertical_fov: float = math.radians(30.0)
    escape_radius: float = 1000.0
    surface: EquatorialSurface | None = None
    horizon_offset: float = 0.0
    _packed: N.Scene | None = field(default=None, init=False, repr=False)

    @classmethod
    def from_oblate(cls, radius: float, polar: float, azimuth: float = 0.0, **kw) -> "Observation":
        chart = kw.get("chart", KerrSchildChart.OUTGOING)
        xyz = oblate_to_cartesian(kw.get("spin", 0.0), chart, radius, polar, azimuth)
        return cls(observer_txyz=(0.0, *xyz), **kw)

    def scene_input(self) -> N.SceneInput:
        s = N.SceneInput()
        s.mass, s.spin, s.charge, s.chart = self.mass, self.spin, self.charge, int(self.chart)
        s.observer_txyz[:] = [float(v) for v in self.observer_txyz]
        s.target_txyz[:] = [float(v) for v in self.target_txyz]
        s.up_hint_xyz[:] = [float(v) for v in self.up_hint_xyz]
        s.measured_frequency = self.measured_frequency
        s.width, s.height, s.vertical_fov = int(self.width), int(self.height), self.vertical_fov
        s.escape_radius = self.escape_radius
        s.has_surface = int(self.surface is not None)
        if self.surface is not None:
            s.surface_inner = self.surface.inner_radius
            s.surface_outer = self.surface.outer_radius
            s.intensity_at_six = self.surface.intensity_at_six
            if self.surface.temperature_at_six is not None:
                s.emission_model = 1
                s.temperature_at_six = self.surface.temperature_at_six
            if self.surface.slab_optical_depth is not None:
                s.has_slab = 1
                s.slab_optical_depth = self.surface.slab_optical_depth
                s.slab_emission = self.surface.slab_emission
                s.slab_temperature = self.surface.slab_temperature
        s.horizon_offset = self.horizon_offset
        return s

    def pack(self) -> N.Scene:
        """glc_scene_pack: validation + tetrad + normalization (raises GlcError on bad input)."""
        out = N.Scene()
        inp = self.scene_input()
        N.check(N.lib().glc_scene_pack(ctypes.byref(inp), ctypes.byref(out)), "glc_scene_pack")
        self._packed = out
        return out

    @property
    def packed(self) -> N.Scene:
        return self._packed if self._packed is not None else self.pack()


class ReferencePolicy:
    """Step-policy presets (policy.rs:28-66) and the frame policies of each precision mode."""

    @staticmethod
    def _preset(preset: int, precision: int) -> N.Policy:
        p = N.Policy()
        N.check(N.lib().glc_policy_default(preset, int(precision), ctypes.byref(p)), "glc_policy_default")
        return p

    @staticmethod
    def regular_v1(precision: int = Precision.FP64) -> N.Policy:
        return ReferencePolicy._preset(0, precision)

    @staticmethod
    def strict_v1(precision: int = Precision.FP64) -> N.Policy:
        return ReferencePolicy._preset(1, precision)

    @staticmethod
    def frame(precision: int = Precision.MIXED, **overrides) -> N.Policy:
        p = ReferencePolicy._preset(2, precision)
        for k, v in overrides.items():
            setattr(p, k, v)
        return p


def _torch():
    import torch

    return torch


class TraceResults:
    """Caller-owned device SoA (glc_results): one 16-byte element per ray per field. The buffers are
    filled with a NaN pattern on the current stream; a trace on another stream (a CUDA graph's, say)
    must be ordered after that fill."""

    def __init__(self, slots: int, device, fields: Iterable[str] = N.RESULT_FIELDS, host: bool = False):
        torch = _torch()
        self.slots = int(slots)
        self.host = host
        self.buffers = {}
        for name in fields:
            nb = N.RESULT_BYTES[name]
            if host:
                t = torch.empty((self.slots, nb), dtype=torch.uint8, pin_memory=True)
            else:
                t = torch.empty((self.slots, nb), dtype=torch.uint8, device=device)
            t.fill_(0xFF)
            self.buffers[name] = t

    def struct(self) -> N.Results:
        r = N.Results()
        for name in N.RESULT_FIELDS:
            t = self.buffers.get(name)
            setattr(r, name, t.data_ptr() if t is not None else None)
        return r

    def numpy(self) -> dict:
        """Decoded fields (host numpy arrays)."""
        out = {}
        b = {k: v.cpu().numpy() if not self.host else v.numpy() for k, v in self.buffers.items()}
        if "code" in b:
            code = b["code"].view(np.uint32).reshape(-1, 4)
            out["termination"] = (code[:, 0] & 0xFF).astype(np.int32)
            out["failure"] = ((code[:, 0] >> 8) & 0xF).astype(np.int32)
            out["candidates"] = ((code[:, 0] >> 12) & 0xF).astype(np.int32)
            out["polar_side"] = ((code[:, 0] >> 16) & 0xF).astype(np.int32) - 1
            out["flags"] = ((code[:, 0] >> 20) & 0xFFF).astype(np.int32)
            out["accepted_steps"] = code[:, 1].astype(np.int64)
            out["rejected_steps"] = code[:, 2].astype(np.int64)
            out["f64_steps"] = code[:, 3].astype(np.int64)
        if "branch" in b:
            br = b["branch"].view(np.int32).reshape(-1, 4)
            out["radial_turnings"], out["equatorial_crossings"] = br[:, 0], br[:, 1]
            out["azimuth_winding"], out["has_turning_radius"] = br[:, 2], br[:, 3]
        pairs = {
            "escape": ("escape_theta", "escape_phi"), "surface": ("source_radius", "source_azimuth"),
            "redshift_time": ("frequency_ratio", "travel_time"),
            "event": ("event_residual", "affine_parameter"),
            "drift_a": ("max_null_residual", "max_energy_drift"),
            "drift_b": ("max_lz_drift", "max_carter_drift"),
            "turning": ("turning_radius", "azimuth_advance"), "position_xy": ("x", "y"),
            "position_zr": ("z", "r"),
        }
        pairs["intensity"] = ("observed_intensity", "emitted_intensity")
        for k, (a, c) in pairs.items():
            if k in b:
                v = b[k].view(np.float64).reshape(-1, 2)
                out[a], out[c] = v[:, 0], v[:, 1]
        if "radiance" in b:
            out["radiance"] = b["radiance"].view(np.float16).reshape(-1, 4).astype(np.float32)
        return out


class Tape:
    """Checkpoints of a forward trace (glc_forward_ckpt); backward() runs the discrete adjoint."""

    def __init__(self, handle, pipeline, slots: int, keepalive):
        self.handle = handle
        self.pipeline = pipeline
        self.slots = slots
        self._keep = keepalive

    def info(self) -> dict:
        rays, cap, nbytes = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint64()
        N.check(N.lib().glc_tape_info(self.handle, ctypes.byref(rays), ctypes.byref(cap), ctypes.byref(nbytes)),
                "glc_tape_info")
        return {"rays": rays.value, "checkpoint_slots": cap.value, "bytes": nbytes.value}

    def backward(self, dl_dobs, stream=None, per_ray_params: bool = True) -> dict:
        """dl_dobs: (slots, 4) float64 dL/d(source radius, g, escape theta, escape phi). Returns device
        tensors ray_momentum (slots, 4) dL/d(p_t, p_x, p_y, p_z), ray_params (slots, 4) and params (4,)
        dL/d(a, Q, inclination, r_obs)."""
        torch = _torch()
        dev = torch.device("cuda", self.pipeline.device)
        dl = torch.as_tensor(dl_dobs).to(device=dev, dtype=torch.float64).contiguous()
        assert tuple(dl.shape) == (self.slots, 4)
        mom = torch.zeros((self.slots, 4), dtype=torch.float64, device=dev)
        rp = torch.zeros((self.slots, 4), dtype=torch.float64, device=dev) if per_ray_params else None
        params = torch.zeros(4, dtype=torch.float64, device=dev)
        g = N.Grads(mom.data_ptr(), rp.data_ptr() if rp is not None else None, params.data_ptr())
        N.check(N.lib().glc_backward(self.handle, ctypes.c_void_p(dl.data_ptr()), ctypes.byref(g),
                                     self.pipeline._stream(stream)), "glc_backward")
        self._last = (dl, mom, rp, params)
        return {"ray_momentum": mom, "ray_params": rp, "params": params}

    def forward_again(self, observation: Observation | None = None, radius: float | None = None,
                      polar: float | None = None, azimuth: float | None = None, results: TraceResults | None = None,
                      stream=None) -> TraceResults:
        """The forward pass again into this tape (glc_forward_ckpt_into), keeping its device memory:
        the same camera and K, with the scene and observer position optionally replaced (an
        optimization step). Returns the new results (written into `results` when given)."""
        a, cam, K = self._request
        if observation is not None:
            a.input = observation.scene_input()
        if radius is not None:
            a.observer_radius = radius
        if polar is not None:
            a.observer_polar = polar
        if azimuth is not None:
            a.observer_azimuth = azimuth
        res = results or TraceResults(self.slots, _torch().device("cuda", self.pipeline.device))
        rs = res.struct()
        N.check(N.lib().glc_forward_ckpt_into(self.pipeline._h, ctypes.byref(a), ctypes.byref(cam), K,
                                              ctypes.byref(rs), self.pipeline._stream(stream), self.handle),
                "glc_forward_ckpt_into")
        return res

    def close(self):
        if self.handle:
            N.lib().glc_tape_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Graph:
    def __init__(self, handle: int, keepalive):
        self.handle = handle
        self._keep = keepalive

    def launch(self, stream=None):
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream()
        N.check(N.lib().glc_graph_launch(self.handle, ctypes.c_void_p(s.cuda_stream)), "glc_graph_launch")

    def close(self):
        if self.handle:
            N.lib().glc_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def image_camera(scene_index: int, width: int, height: int, subpixel=(0.5, 0.5), offset: int = 0,
                 kind: int = N.CAMERA_PINHOLE, region=None) -> N.Camera:
    """An image camera; `region` (a batches.TileRegion) limits the trace to a block of 8x8-pixel
    tiles, written in the whole view's result layout."""
    c = N.Camera()
    c.kind, c.scene_index, c.width, c.height = kind, scene_index, width, height
    c.subpixel_x, c.subpixel_y = subpixel
    c.affine_direction = -1.0
    c.result_offset = offset
    if region is not None:
        c.tile_origin[:] = list(region.origin)
        c.tile_count[:] = list(region.workgroups)
    return c


def raylist_camera(scene_index: int, states_ptr: int, n: int, direction: float, offset: int = 0) -> N.Camera:
    c = N.Camera()
    c.kind, c.scene_index = N.CAMERA_RAYLIST, scene_index
    c.ray_states, c.n_rays, c.affine_direction, c.result_offset = states_ptr, n, direction, offset
    return c


class TracePipeline:
    """Device context (glc_ctx) with its step policy; traces are stream-ordered and asynchronous."""

    def __init__(self, device: int = 0, policy: N.Policy | None = None):
        self.device = device
        h = ctypes.c_void_p()
        N.check(N.lib().glc_create(device, ctypes.byref(h)), "glc_create")
        self._h = h
        if policy is not None:
            self.set_policy(policy)

    # ---- lifecycle
    def close(self):
        if self._h:
            N.lib().glc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- policy and stats
    def set_policy(self, policy: N.Policy) -> None:
        N.check(N.lib().glc_set_policy(self._h, ctypes.byref(policy)), "glc_set_policy")

    @property
    def policy(self) -> N.Policy:
        p = N.Policy()
        N.check(N.lib().glc_get_policy(self._h, ctypes.byref(p)), "glc_get_policy")
        return p

    def stats(self) -> N.LaunchStats:
        s = N.LaunchStats()
        N.check(N.lib().glc_get_stats(self._h, ctypes.byref(s)), "glc_get_stats")
        return s

    # ---- job construction
    @staticmethod
    def _arrays(scenes: Sequence[N.Scene], cameras: Sequence[N.Camera]):
        sa = (N.Scene * len(scenes))(*scenes)
        ca = (N.Camera * len(cameras))(*cameras)
        return sa, ca

    @staticmethod
    def result_slots(scenes, cameras) -> int:
        sa, ca = TracePipeline._arrays(scenes, cameras)
        out = ctypes.c_uint64()
        N.check(N.lib().glc_result_slots(sa, len(scenes), ca, len(cameras), ctypes.byref(out)),
                "glc_result_slots")
        return out.value

    def _stream(self, stream):
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream()
        return ctypes.c_void_p(s.cuda_stream)

    def trace(self, scenes: Sequence[N.Scene], cameras: Sequence[N.Camera], results: TraceResults | None = None,
              stream=None, fields: Iterable[str] = N.RESULT_FIELDS) -> TraceResults:
        torch = _torch()
        if results is None:
            results = TraceResults(self.result_slots(scenes, cameras), torch.device("cuda", self.device), fields)
        sa, ca = self._arrays(scenes, cameras)
        rs = results.struct()
        N.check(N.lib().glc_trace(self._h, sa, len(scenes), ca, len(cameras), ctypes.byref(rs),
                                  self._stream(stream)), "glc_trace")
        return results

    def trace_progressive(self, scenes: Sequence[N.Scene], camera: N.Camera, results: TraceResults | None = None,
                          stream=None, progress=None):
        """Trace one whole-view image camera in tile batches, as the reference's renderer advances a
        frame (Renderer::advance_trace, crates/gravlume-render/src/renderer.rs:470-506, with the
        TraceProgress schedule of renderer/frame.rs:326-420): each batch is a glc_trace of the
        camera's tile region, timed with CUDA events on the stream, and its time rescales the next
        batch's tile budget. Returns the results and the list of (TileRegion, ms)."""
        torch = _torch()
        from .batches import TraceProgress
        from .trace import image_camera as _cam
        if results is None:
            results = TraceResults(self.result_slots(scenes, [camera]), torch.device("cuda", self.device))
        progress = progress or TraceProgress(camera.width, camera.height)
        st = stream if stream is not None else torch.cuda.current_stream()
        done = []
        while (batch := progress.next_batch()) is not None:
            cam = _cam(camera.scene_index, camera.width, camera.height, (camera.subpixel_x, camera.subpixel_y),
                       camera.result_offset, camera.kind, region=batch)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            self.trace(scenes, [cam], results, stream=st)
            e1.record(st)
            progress.submitted(batch)
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            progress.completed(ms)
            done.append((batch, ms))
        return results, done

    def refine_shadow_edges(self, scenes, cameras, primary: TraceResults, stream=None):
        """Coverage per result slot after glc_trace of the same job into `primary`: 1 escape, 0 capture,
        the escaping fraction of four subpixel samples on capture/escape edges, -1 elsewhere."""
        torch = _torch()
        cov = torch.full((primary.slots,), -1.0, dtype=torch.float32, device=torch.device("cuda", self.device))
        sa, ca = self._arrays(scenes, cameras)
        rs = primary.struct()
        N.check(N.lib().glc_refine_shadow_edges(self._h, sa, len(scenes), ca, len(cameras), ctypes.byref(rs),
                                                ctypes.c_void_p(cov.data_ptr()), self._stream(stream)),
                "glc_refine_shadow_edges")
        return cov

    def surface_footprint(self, scenes, cameras, primary: TraceResults, method: str = "quarter_pixel",
                          stream=None):
        """Surface footprints (glc_surface_footprint) after glc_trace of the same job into `primary`:
        a (slots, 8) float64 device tensor of J (dr/dx, dr/dy, darc/dx, darc/dy; M per pixel), major
        and minor singular values, determinant, and the status and parity as int32 pairs in the
        last column's bytes; use `footprint_fields` to split it. method "quarter_pixel" is the
        reference's estimate, "tangent" the forward-mode derivative of the computed trace."""
        torch = _torch()
        m = {"quarter_pixel": FOOTPRINT_QUARTER_PIXEL, "tangent": FOOTPRINT_TANGENT}[method]
        out = torch.empty((primary.slots, 8), dtype=torch.float64, device=torch.device("cuda", self.device))
        sa, ca = self._arrays(scenes, cameras)
        rs = primary.struct()
        N.check(N.lib().glc_surface_footprint(self._h, sa, len(scenes), ca, len(cameras), m, ctypes.byref(rs),
                                              ctypes.c_void_p(out.data_ptr()), self._stream(stream)),
                "glc_surface_footprint")
        return out

    def forward_ckpt(self, observation: Observation, radius: float, polar: float, azimuth: float = 0.0,
                     K: int = 64, states=None, direction: float = -1.0, stream=None):
        """Forward trace with checkpoints every K accepted steps (glc_forward_ckpt). The observer sits
        at oblate (radius, polar, azimuth); the camera is the observation's pinhole view, or the ray
        list `states` (n, 8). Returns (TraceResults, Tape)."""
        torch = _torch()
        a = N.AdjointScene()
        a.input = observation.scene_input()
        a.observer_radius, a.observer_polar, a.observer_azimuth = radius, polar, azimuth
        keep = []
        if states is None:
            cam = image_camera(0, observation.width, observation.height)
            slots = observation.width * observation.height
        else:
            st = torch.as_tensor(np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)).to(
                torch.device("cuda", self.device))
            keep.append(st)
            cam = raylist_camera(0, st.data_ptr(), st.shape[0], direction)
            slots = st.shape[0]
        res = TraceResults(slots, torch.device("cuda", self.device))
        rs = res.struct()
        h = ctypes.c_void_p()
        N.check(N.lib().glc_forward_ckpt(self._h, ctypes.byref(a), ctypes.byref(cam), int(K), ctypes.byref(rs),
                                         self._stream(stream), ctypes.byref(h)), "glc_forward_ckpt")
        tape = Tape(h, self, slots, keep)
        tape._request = (a, cam, int(K))
        return res, tape

    def trace_image(self, observation: Observation, subpixel=(0.5, 0.5), stream=None, **kw) -> TraceResults:
        sc = observation.packed
        return self.trace([sc], [image_camera(0, sc.width, sc.height, subpixel)], stream=stream, **kw)

    def trace_states(self, observation: Observation, states, direction: float = -1.0, stream=None,
                     **kw) -> TraceResults:
        """Trace explicit initial states (t, x, y, z, p_t, p_x, p_y, p_z), GeodesicBatch-style."""
        torch = _torch()
        st = torch.as_tensor(np.ascontiguousarray(states, dtype=np.float64).reshape(-1, 8)).to(
            torch.device("cuda", self.device))
        cam = raylist_camera(0, st.data_ptr(), st.shape[0], direction)
        res = self.trace([observation.packed], [cam], stream=stream, **kw)
        res._states = st  # keep alive until the trace completes
        return res

    def trace_host(self, scenes, cameras, fields: Iterable[str] = N.RESULT_FIELDS) -> TraceResults:
        """End-to-end over host buffers (glc_trace_host): H2D inputs, trace, D2H results."""
        results = TraceResults(self.result_slots(scenes, cameras), None, fields, host=True)
        sa, ca = self._arrays(scenes, cameras)
        rs = results.struct()
        N.check(N.lib().glc_trace_host(self._h, sa, len(scenes), ca, len(cameras), ctypes.byref(rs)),
                "glc_trace_host")
        return results

    def capture_graph(self, scenes, cameras, results: TraceResults, stream) -> Graph:
        sa, ca = self._arrays(scenes, cameras)
        rs = results.struct()
        g = ctypes.c_void_p()
        N.check(N.lib().glc_graph_capture(self._h, sa, len(scenes), ca, len(cameras), ctypes.byref(rs),
                                          ctypes.c_void_p(stream.cuda_stream), ctypes.byref(g)),
                "glc_graph_capture")
        return Graph(g, (results,))

    def autotune(self, scenes, cameras, results: TraceResults | None = None, repeats: int = 1,
                 stream=None) -> N.Policy:
        torch = _torch()
        if results is None:
            results = TraceResults(self.result_slots(scenes, cameras), torch.device("cuda", self.device))
        sa, ca = self._arrays(scenes, cameras)
        rs = results.struct()
        p = self.policy
        N.check(N.lib().glc_autotune(self._h, sa, len(scenes), ca, len(cameras), ctypes.byref(rs),
                                     self._stream(stream), repeats, ctypes.byref(p)), "glc_autotune")
        return p
