"""Regenerate tests/golden/reference_fixtures.json from the reference's versioned TOML fixtures.

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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
