"""Regenerates tests/golden/mc_table_pin.json: SHA-256 digests of the
marching-cubes tables of FluidSim's rebuildSurface
(FluidSim/src/cpu/rebuild-surface.cc:16-21 vertexOffset, :25-29
edgeConnection, :114-639 triangleConnectionTable3D), read as text from the
reference source.  The library keeps the same tables in its own packed form
(simcraft_b200/csrc/sc_mc_table.h); tests/test_surface_cpu.py decodes that
header and compares its digests with these, so the transcription is pinned to
the reference without a second copy of the tables in the repository.

Run (needs the reference source tree): python tests/golden/make_mc_table_pin.py REFERENCE_ROOT
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _initializer(src, name):
    """Text of the brace initializer that follows `name` (comments stripped)."""
    i = src.index(name)
    j = src.index("{", i)
    depth = 0
    for k in range(j, len(src)):
        if src[k] == "{":
            depth += 1
        elif src[k] == "}":
            depth -= 1
            if depth == 0:
                return src[j:k + 1]
    raise ValueError(name)


def _ints(text):
    return [int(x) for x in re.findall(r"-?\d+", text.replace("Vec3i", ""))]


def digests(cases, corners, edges):
    """cases: 256 lists of edge entries (the non-negative entries of each row,
    in order); corners: 8 (x, y, z); edges: 12 (a, b)."""
    import hashlib

    def h(s):
        return hashlib.sha256(s.encode()).hexdigest()

    return {
        "cases": h(";".join(",".join(map(str, c)) for c in cases)),
        "corners": h(";".join(",".join(map(str, c)) for c in corners)),
        "edges": h(";".join(",".join(map(str, e)) for e in edges)),
    }


def main(ref_root):
    path = os.path.join(ref_root, "FluidSim", "src", "cpu", "rebuild-surface.cc")
    src = re.sub(r"//[^\n]*", "", open(path).read())
    vo = _ints(_initializer(src, "vertexOffset ="))
    ec = _ints(_initializer(src, "edgeConnection["))
    tt = _ints(_initializer(src, "triangleConnectionTable3D["))
    assert len(vo) == 24 and len(ec) == 24 and len(tt) == 256 * 16
    cases = [[e for e in tt[16 * m:16 * m + 16] if e >= 0] for m in range(256)]
    corners = [tuple(vo[3 * i:3 * i + 3]) for i in range(8)]
    edges = [tuple(ec[2 * i:2 * i + 2]) for i in range(12)]
    out = digests(cases, corners, edges)
    out["source"] = "FluidSim/src/cpu/rebuild-surface.cc:16-21,25-29,114-639"
    with open(os.path.join(HERE, "mc_table_pin.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    print(out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_mc_table_pin.py REFERENCE_ROOT (the SimCraft source tree)")
    main(sys.argv[1])
