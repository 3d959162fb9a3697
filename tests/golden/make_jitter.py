"""Extract the aa_fill sample offsets from the reference source as a fixture.

    python tests/golden/make_jitter.py path/to/reference

Reads the HALTON2 / HALTON3 tables of crates/gpu/src/fill.rs (the jitter of
the reference's aa_fill operator) as text and writes aa_fill_jitter.json:
the 64 x and 64 y offsets exactly as the reference spells them. The oracle
and the library generate these tables themselves; tests/test_fill_ops.py
checks their f32 values against this fixture bit for bit.
"""

import json
import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def table(src: str, name: str) -> list[str]:
    m = re.search(rf"const {name}: \[f32; 64\] = \[(.*?)\];", src, re.S)
    body = re.sub(r"//[^\n]*", "", m.group(1))
    vals = [v.strip().replace("_", "") for v in body.split(",") if v.strip()]
    assert len(vals) == 64, (name, len(vals))
    return vals


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_jitter.py path/to/reference (the rasterrocket source tree)")
    ref = Path(sys.argv[1])
    src = (ref / "crates/gpu/src/fill.rs").read_text()
    out = {"source": "crates/gpu/src/fill.rs HALTON2 / HALTON3", "x": table(src, "HALTON2"),
           "y": table(src, "HALTON3")}
    (HERE / "aa_fill_jitter.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
