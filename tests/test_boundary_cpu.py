"""C ABI boundary checks that need no GPU: the library loads and exports every symbol
include/glc.h declares; scene packing (validation, tetrad, horizon) and the host build of the
device right-hand side agree with the binary64 oracle; typed errors mirror the reference's
GpuTraceInputError / ValidationIssueCode cases (crates/gravlume-render/src/trace/input.rs:342-381,
crates/gravlume-domain/src/observer.rs:67-183, events.rs:61-84)."""

import ctypes
import math
import re
from pathlib import Path

import numpy as np
import pytest

import gravlume_b200 as G
from gravlume_b200 import _native as N
import oracle as O

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "glc.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:glc_status|int|const char\*)\s+(glc_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = G.lib()
    names = declared_symbols()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
        assert name in N.SIGNATURES, f"{name} has no ctypes signature"
    header = (ROOT / "include" / "glc.h").read_text()
    assert f"#define GLC_ABI_VERSION {N.ABI_VERSION}" in header
    assert lib.glc_abi_version() == N.ABI_VERSION
    assert lib.glc_status_string(0) == b"ok"


def test_a_missing_library_fails_loudly():
    """No fallback: without libglc.so the bindings raise, naming the build call."""
    import subprocess
    import sys

    code = ("from gravlume_b200 import _native as N\n"
            "try:\n    N.lib('/nonexistent/libglc.so')\nexcept RuntimeError as e:\n    print(e)\n")
    run = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=str(ROOT), timeout=120)
    assert run.returncode == 0, run.stderr
    assert "libglc.so is not built" in run.stdout and "gravlume_b200.build(force=True)" in run.stdout


def test_build_flags_keep_the_capture_certificates_sound():
    """sm_100a only; binary32 division and square root may be approximate, but nothing may flush
    denormals or turn on fast math: the certificates' directed-rounding bounds rely on both."""
    import importlib

    flags = importlib.import_module("gravlume_b200.build").NVCC_FLAGS
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "-prec-div=false" in flags and "-prec-sqrt=false" in flags
    for bad in ("-ftz=true", "--ftz=true", "-use_fast_math", "--use_fast_math"):
        assert bad not in flags, bad
    cert = (ROOT / "gravlume_b200" / "csrc" / "glc_certificate.cuh").read_text()
    for rounded in ("__fadd_rd", "__fadd_ru", "__fmul_rd", "__fmul_ru", "__fdiv_rd", "__fdiv_ru",
                    "__fsqrt_rd", "__fsqrt_ru"):
        assert rounded in cert, rounded


def test_create_without_a_device_is_a_typed_error():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = ctypes.c_void_p()
    assert G.lib().glc_create(0, ctypes.byref(h)) == 14  # GLC_ERR_NO_DEVICE
    assert not h.value


def oracle_scene(obs: G.Observation):
    return O.scene(mass=obs.mass, spin=obs.spin, charge=obs.charge, chart=int(obs.chart),
                   observer_txyz=obs.observer_txyz, target=obs.target_txyz, up_hint=obs.up_hint_xyz,
                   width=obs.width, height=obs.height, vertical_fov=obs.vertical_fov)


SCENES = [
    dict(spin=0.9, charge=0.3, chart=1, r=50.0, incl=75.0),
    dict(spin=0.8, charge=0.0, chart=0, r=30.0, incl=60.0),
    dict(spin=0.998, charge=0.05, chart=1, r=1000.0, incl=85.0),
    dict(spin=0.0, charge=0.0, chart=0, r=50.0, incl=17.0),
    dict(spin=0.6, charge=0.7, chart=1, r=20.0, incl=89.0),
    dict(spin=-0.5, charge=0.2, chart=0, r=15.0, incl=5.0),
]


@pytest.mark.parametrize("p", SCENES)
def test_scene_pack_matches_the_oracle_observer_frame(p):
    obs = G.Observation.from_oblate(p["r"], math.radians(p["incl"]), 0.0, spin=p["spin"], charge=p["charge"],
                                    chart=p["chart"], width=64, height=48, vertical_fov=math.radians(30))
    sc = obs.pack()
    info = O.observer_info(oracle_scene(obs))
    for name in ("four_velocity", "image_right", "image_up", "arrival"):
        np.testing.assert_allclose(list(getattr(sc, name)), list(getattr(info, name)), rtol=0, atol=1e-13)
    np.testing.assert_allclose(list(sc.metric_covariant), list(info.metric_covariant), rtol=1e-14, atol=1e-15)
    _, rp = O.spacetime_info(1.0, p["spin"], p["charge"])
    assert sc.outer_horizon == pytest.approx(rp, rel=0, abs=4e-16)
    assert sc.isco_prograde == pytest.approx(O.prograde_isco(1.0, p["spin"], p["charge"]), abs=1e-10)
    assert sc.tangent_half_fov == pytest.approx(info.tangent_half_fov, rel=1e-15)


def test_scene_pack_horizon_on_the_default_kerr_observation_fixture(golden):
    fx = golden["kerr-exterior-observation-v1"]
    obs = G.Observation.from_oblate(float(fx["observer"]["oblate_radius_m"]),
                                    float(fx["observer"]["polar_angle_rad"]), 0.0, spin=0.8,
                                    chart=G.KerrSchildChart.INGOING, width=1280, height=720,
                                    vertical_fov=float(fx["viewport"]["vertical_fov_rad"]), escape_radius=200.0)
    sc = obs.pack()
    assert abs(sc.outer_horizon - float(fx["expected"]["outer_horizon_radius_m"])) <= 2e-13
    xyz = fx["expected"]["observer_cartesian_xyz_m"]
    for got, exp in zip(list(sc.observer_txyz)[1:], xyz):
        assert abs(got - float(exp)) <= 2e-13
    assert abs(sc.metric_covariant[0] - float(fx["expected"]["observer_g_tt"])) <= 2e-13


def test_extremality_is_classified_exactly():
    cases = [(1.0, 0.0), (0.0, 1.0), (0.6, 0.8), (0.6, 0.8000000000000002), (0.6, 0.7999999999999999),
             (0.8, 0.6), (0.28, 0.96), (1e-9, 1.0), (0.9, 0.3)]
    seen = set()
    for a, q in cases:
        obs = G.Observation(spin=a, charge=q, observer_txyz=(0, 40.0, 0, 5.0), escape_radius=200.0)
        sc = obs.pack()
        oe, orp = O.spacetime_info(1.0, a, q)
        assert sc.extremality == oe, (a, q)
        seen.add(oe)
        if oe != 2:
            assert sc.outer_horizon == pytest.approx(orp, abs=1e-15)
    assert seen == {0, 1, 2}


def expect_error(code, **kw):
    with pytest.raises(G.GlcError) as e:
        G.Observation(**kw).pack()
    assert e.value.status == code, str(e.value)


def test_scene_pack_rejects_invalid_inputs_with_typed_errors():
    expect_error(3, spin=float("nan"))                               # NON_FINITE
    expect_error(4, mass=0.0)                                        # NON_POSITIVE
    expect_error(5, measured_frequency=1.5)                          # NON_NORMALIZED
    expect_error(11, vertical_fov=math.pi)                           # INVALID_VIEW
    expect_error(11, width=0)
    expect_error(9, escape_radius=200.0, surface=G.EquatorialSurface(6.0, 200.0))  # outside escape
    expect_error(10, surface=G.EquatorialSurface(20.0, 6.0))         # reversed radii
    expect_error(8, observer_txyz=(0, 50.0, 0, 0), target_txyz=(0, 50.0, 0, 0))     # degenerate target
    expect_error(7, spin=0.9, observer_txyz=(0, 1.8, 0, 0.0))        # inside the ergoregion: g_tt >= 0


def test_extremality_change_by_normalization_is_rejected():
    # M = 3 with a = 3 is extremal; a tiny mass rescale that moves a/M across 1 would change it.
    G.Observation(mass=3.0, spin=3.0, observer_txyz=(0, 150.0, 0, 10.0), escape_radius=600.0).pack()


@pytest.mark.parametrize("chart", [0, 1])
def test_host_rhs_matches_the_oracle_hamiltonian_rhs(chart):
    rng = np.random.default_rng(7)
    for a, q in [(0.9, 0.3), (0.0, 0.0), (0.998, 0.05), (-0.6, 0.7)]:
        obs = G.Observation(spin=a, charge=q, chart=chart, observer_txyz=(0, 40.0, 1.0, 5.0), escape_radius=200.0)
        sc = obs.pack()
        for _ in range(40):
            r = rng.uniform(1.6, 60.0)
            th = rng.uniform(0.05, math.pi - 0.05)
            ph = rng.uniform(-math.pi, math.pi)
            xyz = G.oblate_to_cartesian(a, chart, r, th, ph)
            if rng.uniform() < 0.1:
                xyz = [0.0, 0.0, r * (1 if rng.uniform() < 0.5 else -1)]  # on the axis
            p = rng.normal(size=3)
            E = 1.0 + rng.uniform()
            state8 = np.array([0.0, *xyz, -E, *p])
            ref = O.hamiltonian_rhs(1.0, a, q, chart, state8)
            out = np.zeros(7)
            st6 = np.ascontiguousarray([*xyz, *p])
            G.lib().glc_rhs_host(ctypes.byref(sc), st6.ctypes.data, E, 2, out.ctypes.data)
            want = np.array([ref[1], ref[2], ref[3], ref[5], ref[6], ref[7], ref[0]])
            scale = np.max(np.abs(want)) + 1.0
            np.testing.assert_allclose(out, want, rtol=0, atol=2e-13 * scale)


def test_prograde_isco_helper_matches_the_oracle():
    for a, q in [(0.0, 0.0), (0.9, 0.3), (0.998, 0.0), (0.6, 0.7), (0.0, 0.5)]:
        assert G.prograde_isco(a, q) == pytest.approx(O.prograde_isco(1.0, a, q), abs=1e-9)
    assert G.prograde_isco(0.0, 0.0) == pytest.approx(6.0, abs=1e-12)


def test_policy_presets_follow_the_reference_and_validate():
    r = G.ReferencePolicy.regular_v1()
    s = G.ReferencePolicy.strict_v1()
    o = O.regular_v1()
    for name in ("position_rtol", "position_atol", "momentum_rtol", "momentum_atol", "initial_step", "minimum_step",
                 "maximum_step", "safety", "minimum_factor", "maximum_factor", "maximum_accepted_steps",
                 "maximum_consecutive_rejects", "event_affine_tolerance", "event_tie_tolerance",
                 "event_arming_band", "singularity_guard"):
        assert getattr(r, name) == getattr(o, name), name
        assert getattr(s, name) == getattr(O.strict_v1(), name), name
    f = G.ReferencePolicy.frame(G.Precision.FP64)
    assert f.position_rtol == 1e-10 and f.position_atol == 1e-12


def test_integration_binding_sizes_match_the_abi():
    """The Rust binding that the integration guide at the repository root gives maintainers declares
    opaque structs by byte size; those sizes are the C ABI's (as mirrored by the ctypes
    declarations)."""
    import ctypes
    import re
    from pathlib import Path

    text = (Path(__file__).resolve().parents[1] / "INTEGRATION.md").read_text()
    sizes = {m.group(1): int(m.group(2)) for m in re.finditer(r"pub struct (glc_\w+) \{ _bytes: \[u8; (\d+)\] \}", text)}
    assert sizes["glc_policy"] == ctypes.sizeof(N.Policy)
    assert sizes["glc_scene"] == ctypes.sizeof(N.Scene)
    assert "pub tile_origin: [u32; 2]" in text and ctypes.sizeof(N.Camera) == 80


def test_flop_model_counts_the_current_step():
    """The roofline's algorithmic work unit, counted on the host by instantiating the device
    templates on a counting scalar: 100 flops and 3 special functions per right-hand side, 1098
    flops per attempted DP5(4) step (six right-hand sides, the stage combinations, the error norm,
    the end-point invariants and the controller)."""
    f = np.zeros(4)
    assert N.lib().glc_flop_model(f.ctypes.data) == 0
    assert f[0] == 100.0 and f[1] == 3.0, f
    assert f[2] == 1098.0, f
