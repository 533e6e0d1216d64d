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


def main(reference_root: str) -> None:
    base = Path(reference_root) / "crates" / "gravlume-reference" / "fixtures"
    out = {}
    for rel in FIXTURES:
        doc = tomllib.loads((base / rel).read_text())
        doc["_source"] = f"crates/gravlume-reference/fixtures/{rel}"
        out[doc["id"]] = doc
    target = Path(__file__).with_name("reference_fixtures.json")
    target.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {target} ({len(out)} fixtures)")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
