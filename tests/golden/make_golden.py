"""Regenerate tests/golden/reference_fixtures.json from the reference's versioned TOML fixtures,
and tests/golden/gpu_gate_cases.json from the reference's GPU-against-CPU tests.

The reference pins its CPU oracle with strict TOML known-answer fixtures
(crates/gravlume-reference/fixtures/v1/*.toml and fixtures/v2/kerr-surface-observable.toml,
accepted by crates/gravlume-reference/src/fixture.rs:228-325 and fixture/v1.rs:321-366). This
script extracts their inputs, expected values and tolerances, as the decimal strings they are
stored in, into one JSON file that travels with the tests. Run it where the reference checkout is
available:

    python tests/golden/make_golden.py /path/to/gravlume
"""

from __future__ import annotations

import json
import sys
import tomllib
from pathlib import Path

FIXTURES = [
    "v1/schwarzschild-scatter-b6.toml",
    "v1/schwarzschild-scatter-near-critical.toml",
    "v1/schwarzschild-capture-near-critical.toml",
    "v1/default-kerr-observation.toml",
    "v2/kerr-surface-observable.toml",
]


# Known answers written inline in the reference's unit tests of the surface radiation model
# (crates/gravlume-reference/src/radiation.rs, mod tests): the test whose name matches, the
# temperature and bolometric intensity it evaluates, and its expected band intensities and tolerance.
RADIATION_TESTS = {
    "six_thousand_kelvin_bands_match_the_independent_high_precision_oracle": "blackbody-bands-6000K",
    "low_temperature_diluted_spectrum_preserves_representable_bands": "blackbody-bands-220K-diluted",
    "dimensionless_planck_integral_closes_stefan_boltzmann_normalization": "planck-integral-normalization",
}


def radiation_known_answers(reference_root: str) -> dict:
    import re

    rel = "crates/gravlume-reference/src/radiation.rs"
    src = (Path(reference_root) / rel).read_text()
    out = {}
    for test, fid in RADIATION_TESTS.items():
        body = src[src.index(f"fn {test}()"):]
        body = body[: body.index("\n    }\n")]
        numbers = [n.replace("_", "") for n in re.findall(r"[-+]?\d[\d_]*\.?[\d_]*(?:e[-+]?\d+)?", body)]
        entry = {"id": fid, "_source": f"{rel} ({test})"}
        if fid == "planck-integral-normalization":
            call = re.search(r"integrate_planck_kernel\(([^,]+),\s*([^)]+)\)", body)
            entry["interval"] = [call.group(1).strip(), call.group(2).strip()]
            entry["expected"] = "pi^4/15"
            entry["tolerance_abs"] = re.search(r"epsilon = ([0-9.e-]+)", body).group(1)
        else:
            call = re.search(r"blackbody_band_intensities\(([^,]+),\s*([^)]+)\)", body)
            entry["bolometric_intensity"] = call.group(1).strip().replace("_", "")
            entry["temperature_kelvin"] = call.group(2).strip().replace("_", "")
            exp = re.search(r"let expected = \[(.*?)\];", body, re.S).group(1)
            entry["expected_bands_rgb"] = [v.strip().replace("_", "") for v in exp.split(",") if v.strip()]
            tol = re.search(r"epsilon = ([0-9.e-]+)( \* expected)?", body)
            entry["tolerance"] = tol.group(1)
            entry["tolerance_is_relative"] = bool(tol.group(2))
        out[fid] = entry
    return out


# The reference's GPU-against-CPU gates (crates/gravlume-render/src/gpu_trace_tests.rs and
# gpu_trace_tests/surface.rs): the image samples, scenes and tolerances they check the WGSL RK4
# kernel with. The scene helpers are restated here, cited; the sample tables and tolerances are
# read from the test source.
_ANGLES = {"FRAC_PI_2": "pi/2", "FRAC_PI_3": "pi/3", "FRAC_PI_4": "pi/4"}


def gpu_gate_cases(reference_root: str) -> dict:
    import re

    root = Path(reference_root) / "crates" / "gravlume-render" / "src"
    rel = "crates/gravlume-render/src/gpu_trace_tests.rs"
    src = (root / "gpu_trace_tests.rs").read_text()
    test = "headless_gpu_regular_matrix_matches_reference_termination_and_escape_direction"
    body = src[src.index(f"fn {test}()"):]
    body = body[: body.index("\n}\n")]
    extent = re.search(r"default_observation\((\d+),\s*(\d+)\)", body)
    samples = [[int(x), int(y)] for x, y in re.findall(r"sample\(&observation,\s*(\d+),\s*(\d+),", body)]
    regular = {
        "_source": f"{rel} ({test}; observation_at_scale, observation_with_time)",
        "width": int(extent.group(1)), "height": int(extent.group(2)),
        # observation_at_scale (mass 1): a = 0.8 M, Q = 0, outgoing chart, observer at oblate
        # (30 M, pi/3, 0) looking at the origin with +z up, omega = 1, vertical FOV pi/4; the
        # CPU side traces ObservationTracer::baseline_v1 (escape at 200 M) with regular_v1.
        "spin": 0.8, "charge": 0.0, "chart": "outgoing", "observer_oblate": [30.0, "pi/3", 0.0],
        "vertical_fov": "pi/4", "escape_radius": 200.0,
        "samples": samples,
        "escape_angle_rad": float(re.search(r"angular_error <= ([0-9.e-]+)", body).group(1)),
        "event_residual": float(re.search(r"event_residual <= ([0-9.e-]+)", body).group(1)),
        "travel_time_m": float(re.search(r"travel_time_error <= ([0-9.e-]+)", body).group(1)),
        "drift_limit": 0.05,  # INVARIANT_DRIFT_LIMIT (crates/gravlume-render/src/trace/input.rs:13)
    }
    rel_s = "crates/gravlume-render/src/gpu_trace_tests/surface.rs"
    ssrc = (root / "gpu_trace_tests" / "surface.rs").read_text()
    table = ssrc[ssrc.index("const SURFACE_BRANCH_PROFILES"):]
    table = table[: table.index("\n];\n")]
    profiles = []
    for block in table.split("SurfaceBranchProfile {")[1:]:
        fov = re.search(r"vertical_fov: std::f64::consts::(\w+)", block).group(1)
        profiles.append({
            "label": re.search(r'label: "([^"]+)"', block).group(1),
            "spin": float(re.search(r"spin: ([-0-9.]+)", block).group(1)),
            "charge": float(re.search(r"charge: ([-0-9.]+)", block).group(1)),
            "observer_radius": float(re.search(r"observer_radius: ([0-9.]+)", block).group(1)),
            "vertical_fov": _ANGLES[fov],
            "samples": [[int(x), int(y)] for x, y in re.findall(r"\((\d+),\s*(\d+)\)", block)],
        })
    fn = ssrc[ssrc.index("fn assert_surface_branch_profile"):]
    ext = re.search(r"vertical_fov,\s*(\d+),\s*(\d+),", fn)
    emit = re.search(r"inverse_cube_bolometric_v1\(([0-9.]+),\s*([0-9.]+),", fn)
    surface = {
        "_source": f"{rel_s} (gpu_surface_branches_match_fixed_reference_samples); "
                   f"{rel} (transfer_profile_extent)",
        # transfer_profile_extent: outgoing chart, observer at oblate (r, pi/3, 0) looking at the
        # origin with +z up, omega = 1; vacuum inverse-cube bolometric surface; escape at 200 M.
        "width": int(ext.group(1)), "height": int(ext.group(2)), "observer_polar": "pi/3",
        "surface": [float(emit.group(1)), float(emit.group(2))], "escape_radius": 200.0,
        "profiles": profiles,
    }
    return {"regular_matrix": regular, "surface_branches": surface}


def main(reference_root: str) -> None:
    base = Path(reference_root) / "crates" / "gravlume-reference" / "fixtures"
    out = {}
    for rel in FIXTURES:
        doc = tomllib.loads((base / rel).read_text())
        doc["_source"] = f"crates/gravlume-reference/fixtures/{rel}"
        out[doc["id"]] = doc
    out.update(radiation_known_answers(reference_root))
    target = Path(__file__).with_name("reference_fixtures.json")
    target.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {target} ({len(out)} fixtures)")
    gates = Path(__file__).with_name("gpu_gate_cases.json")
    gates.write_text(json.dumps(gpu_gate_cases(reference_root), indent=1) + "\n")
    print(f"wrote {gates}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of a romeoahmed/gravlume checkout>")
    main(sys.argv[1])
