"""Generates the golden fixtures under tests/golden/ from the reference crate's own
test sources (meshless_voronoi 0.7.2).  Usage:

    python tests/golden/make_fixtures.py <path of the reference crate's checkout>

The outputs are committed, so the tests never read the reference at run time.

* non_perturbed_z.json -- the 40-point thin-box fixture of test_non_perturbed_z
  (src/voronoi.rs:1248-1296): anchor, width and generators, parsed as text.
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

NUM = r"(-?[0-9.]+(?:e-?[0-9]+)?)"
VEC = re.compile(r"DVec3::new\(\s*" + NUM + r",\s*" + NUM + r",\s*" + NUM + r"\s*\)")


def non_perturbed_z(ref: str):
    src = open(os.path.join(ref, "src", "voronoi.rs")).read()
    start = src.index("fn test_non_perturbed_z")
    body = src[start:src.index("consistency_check", start)]
    vecs = [[float(a), float(b), float(c)] for a, b, c in VEC.findall(body)]
    anchor, width, points = vecs[0], vecs[1], vecs[2:]
    assert len(points) == 40, len(points)
    return {"source": "src/voronoi.rs:1248-1296 (test_non_perturbed_z)",
            "anchor": anchor, "width": width, "generators": points,
            "dimensionality": 3, "periodic": False}


def main(argv):
    if len(argv) != 2:
        raise SystemExit("usage: make_fixtures.py <reference crate checkout>")
    fx = non_perturbed_z(argv[1])
    with open(os.path.join(HERE, "non_perturbed_z.json"), "w") as f:
        json.dump(fx, f, indent=1)
    print("wrote non_perturbed_z.json with", len(fx["generators"]), "generators")


if __name__ == "__main__":
    main(sys.argv)
