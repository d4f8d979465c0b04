"""Regenerates the golden fixtures of tests/golden from the RTK reference tree.

geometry_kat.json: the two projections and 3x4 matrices published in RTK's
documentation/docs/Geometry.md (XML example, SID 1000 / SDD 1536), parsed from
the document itself.  geometry_example.xml: that XML example verbatim.

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


def geometry_md_xml(path: str) -> str:
    """The XML example of the document, verbatim (a file the geometry reader
    must accept: version 3, global SID/SDD/radius, per-projection matrices)."""
    txt = open(path).read()
    return re.search(r"(<\?xml.*?</RTKThreeDCircularGeometry>)", txt, flags=re.S).group(1) + "\n"


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of an RTK source tree>")
    ref = sys.argv[1]
    here = os.path.dirname(os.path.abspath(__file__))
    md = os.path.join(ref, "documentation", "docs", "Geometry.md")
    kat = parse_geometry_md(md)
    with open(os.path.join(here, "geometry_kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    print("wrote geometry_kat.json with", len(kat["projections"]), "projections")
    with open(os.path.join(here, "geometry_example.xml"), "w") as f:
        f.write(geometry_md_xml(md))
    print("wrote geometry_example.xml")


if __name__ == "__main__":
    main()
