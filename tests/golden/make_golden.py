"""Regenerates the golden fixtures of tests/golden from the RTK reference tree.

geometry_kat.json: the two projections and 3x4 matrices published in RTK's
documentation/docs/Geometry.md (XML example, SID 1000 / SDD 1536), parsed from
the document itself.

Run inside the development container (the reference tree is not available
where the tests run):  python tests/golden/make_golden.py /path/to/RTK
"""
from __future__ import annotations

import json
import os
import re
import sys


def parse_geometry_md(path: str) -> dict:
    txt = open(path).read()
    sid = float(re.search(r"<SourceToIsocenterDistance>([^<]+)<", txt).group(1))
    sdd = float(re.search(r"<SourceToDetectorDistance>([^<]+)<", txt).group(1))
    projs = []
    for block in re.findall(r"<Projection>(.*?)</Projection>", txt, flags=re.S):
        def val(tag):
            m = re.search(rf"<{tag}>([^<]+)<", block)
            return float(m.group(1)) if m else 0.0

        mat = [float(x) for x in re.search(r"<Matrix>(.*?)</Matrix>", block, flags=re.S).group(1).split()]
        projs.append({"gantry_angle": val("GantryAngle"), "proj_offset_x": val("ProjectionOffsetX"),
                      "proj_offset_y": val("ProjectionOffsetY"), "matrix": mat})
    return {"source": "documentation/docs/Geometry.md", "sid": sid, "sdd": sdd, "projections": projs}


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    here = os.path.dirname(os.path.abspath(__file__))
    kat = parse_geometry_md(os.path.join(ref, "documentation", "docs", "Geometry.md"))
    with open(os.path.join(here, "geometry_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    print("wrote geometry_kat.json with", len(kat["projections"]), "projections")


if __name__ == "__main__":
    main()
