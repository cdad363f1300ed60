"""CPU restatement of the reference's on-disk formats (test infrastructure, not the
product).  Only tests/ import this module.

* vtk_text: the legacy VTK snapshot as writeGeometryToVTK writes it
  (delta/core/io/write.cpp:226-306), for bodies given as (3, 3*nT) vertex arrays;
* mbfcp_spheres: what readmbfcp (delta/core/io/read.cpp:345-546) extracts from a .mbfcp
  text: the material block's values (std::stof at the fixed offsets), the BODIES count and
  each SPHERES body's (id, centre, radius) from the fixed-offset substrings.
"""
from __future__ import annotations

import numpy as np


def vtk_text(bodies) -> str:
    nv = sum(b.shape[1] for b in bodies)
    nf = nv // 3
    out = ["# vtk DataFile Version 2.0\nOutput vtk file\nASCII\n\nDATASET UNSTRUCTURED_GRID\n",
           f"POINTS {nv} double\n"]
    for b in bodies:
        for j in range(b.shape[1]):
            out.append("%.5f %.5f %.5f\n" % (b[0, j], b[1, j], b[2, j]))
    out.append(f"\nCELLS {nf} {4 * nf}\n")
    for f in range(nf):
        out.append(f"3 {3 * f} {3 * f + 1} {3 * f + 2}\n")
    out.append(f"\nCELL_TYPES {nf}\n")
    out.append("5\n" * nf)
    return "".join(out)


def _stof(s: str) -> float:
    """std::stof: leading whitespace, the longest float prefix, rounded to float32."""
    import re

    m = re.match(r"\s*([+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?))", s)
    if not m:
        raise ValueError(s)
    return float(np.float32(float(m.group(1))))


def _stod(s: str) -> float:
    import re

    m = re.match(r"\s*([+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?))", s)
    if not m:
        raise ValueError(s)
    return float(m.group(1))


def _stoi(s: str) -> int:
    import re

    m = re.match(r"\s*([+-]?\d+)", s)
    if not m:
        raise ValueError(s)
    return int(m.group(1))


def mbfcp_spheres(text: str) -> dict:
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    out = {"bodies": 0, "materials": None, "spheres": []}
    i = 0

    def nxt():
        nonlocal i
        line = lines[i] if i < len(lines) else ""
        i += 1
        return line

    while i < len(lines):
        line = nxt()
        if not line:
            continue
        if "SURFACE_MATERIALS:" in line:
            ls = [nxt() for _ in range(19)]
            out["materials"] = {"friction": _stof(ls[3][10:]), "spring": _stof(ls[5][8:]),
                                "dashpot": _stof(ls[6][8:]), "density": _stof(ls[13][9:]),
                                "gravity": [_stof(ls[16 + k][10:]) for k in range(3)]}
            line = ls[18]
        if "BODIES:" in line:
            out["bodies"] = _stoi(line[8:])
        if "ID:" in line and line.find("SURFID:") != 0:
            ident = _stoi(line[3:])
            for _ in range(5):
                line = nxt()
            if "SPHERES:" in line:
                line = nxt()
                c = [_stod(line[8 + 6 * k:12 + 6 * k]) for k in range(3)]
                line = nxt()
                out["spheres"].append((ident, c, _stod(line[8:12])))
    return out
