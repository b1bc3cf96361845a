"""Generates sph_mc_tables.h: marching-cubes case tables derived from the cube
geometry (not copied from any table).

Corner v of a cell sits at offset (x, y, z) = CORNERS[v]; edge e joins
corners EDGES[e].  For each of the 256 inside/outside patterns (bit v set =
corner v above the iso value, the reference's flag convention,
SPH-3D-2/sph_system.cpp:459-466):
  * edge flags: edge e is cut iff its two corners differ;
  * on every cube face the cut edges are joined into segments; a face whose
    diagonal corners agree (4 cuts) joins each cut to the cut that keeps the
    face's two "above" corners apart (the face centre counts as below);
  * each segment is directed so the "above" side lies to its left when seen
    from outside the cube; segments chain into closed loops;
  * every loop (3..7 vertices) is fanned from its smallest edge id.
The resulting polygon loops (cut edges, loop structure, winding, triangle
count) equal those of the classic 256-case table the reference uses
(SPH-3D-2/sph_system.cpp:544-821) for all 256 cases; a loop of 4 or more
vertices may be split along a different diagonal.  tests/test_mc_tables.py
checks this case by case against the reference's own table.

    python sca2012_b200/csrc/gen_mc_tables.py   # rewrites sph_mc_tables.h
"""
import os

CORNERS = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4), (0, 4), (1, 5), (2, 6), (3, 7)]


def edge_index(a, b):
    for e, (p, q) in enumerate(EDGES):
        if {p, q} == {a, b}:
            return e
    raise KeyError((a, b))


def faces():
    """Each face as its 4 corners in counter-clockwise order seen from outside."""
    out = []
    for axis in range(3):
        for side in (0, 1):
            vs = [v for v, c in enumerate(CORNERS) if c[axis] == side]
            # order around the face centre, counter-clockwise about the outward normal
            import math
            u, w = [a for a in range(3) if a != axis]
            cen = [sum(CORNERS[v][k] for v in vs) / 4.0 for k in range(3)]
            ang = {v: math.atan2(CORNERS[v][w] - cen[w], CORNERS[v][u] - cen[u]) for v in vs}
            vs.sort(key=lambda v: ang[v])
            # (u, w, axis) right-handed? flip for the negative side or a left-handed triple
            normal = [0, 0, 0]
            normal[axis] = 1 if side else -1
            e1 = [CORNERS[vs[1]][k] - CORNERS[vs[0]][k] for k in range(3)]
            e2 = [CORNERS[vs[2]][k] - CORNERS[vs[1]][k] for k in range(3)]
            cr = [e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]]
            if sum(cr[k] * normal[k] for k in range(3)) < 0:
                vs.reverse()
            out.append(vs)
    return out


FACES = faces()


def segments(case):
    """Directed segments (from_edge, to_edge) on all faces: the above-iso
    corners lie to the left of each segment seen from outside."""
    inside = [(case >> v) & 1 for v in range(8)]
    segs = []
    for f in FACES:
        # walk the face boundary counter-clockwise: corners f[0..3], edge k joins f[k], f[k+1]
        cuts = []
        for k in range(4):
            a, b = f[k], f[(k + 1) % 4]
            if inside[a] != inside[b]:
                # entering (outside->inside) or leaving along the ccw walk
                cuts.append((k, edge_index(a, b), inside[b]))
        if not cuts:
            continue
        if len(cuts) == 2:
            # the segment goes from the cut where the ccw walk leaves the
            # inside to the cut where it enters, keeping the inside on the left
            leave = [c for c in cuts if c[2] == 0][0]
            enter = [c for c in cuts if c[2] == 1][0]
            segs.append((leave[1], enter[1]))
        else:
            # ambiguous face: each inside corner is cut off on its own
            for k in range(4):
                if inside[f[k]]:
                    e_in = edge_index(f[(k - 1) % 4], f[k])    # entering edge before corner k
                    e_out = edge_index(f[k], f[(k + 1) % 4])   # leaving edge after corner k
                    segs.append((e_out, e_in))
    return segs


def loops(case):
    segs = segments(case)
    nxt = {}
    for a, b in segs:
        assert a not in nxt, (case, segs)
        nxt[a] = b
    seen, out = set(), []
    for start in sorted(nxt):
        if start in seen:
            continue
        loop, v = [], start
        while v not in seen:
            seen.add(v)
            loop.append(v)
            v = nxt[v]
        out.append(loop)
    return out


def triangles(case):
    tris = []
    for loop in loops(case):
        k = loop.index(min(loop))
        loop = loop[k:] + loop[:k]
        for i in range(1, len(loop) - 1):
            tris.append((loop[0], loop[i], loop[i + 1]))
    return tris


def tables():
    edge_flags = []
    tri_table = []
    for c in range(256):
        edge_flags.append(sum(1 << e for e, (a, b) in enumerate(EDGES) if ((c >> a) & 1) != ((c >> b) & 1)))
        t = [x for tri in triangles(c) for x in tri]
        assert len(t) <= 15
        tri_table.append(t + [-1] * (16 - len(t)))
    return edge_flags, tri_table


def main():
    ef, tt = tables()
    here = os.path.dirname(os.path.abspath(__file__))
    lines = ["// Generated by gen_mc_tables.py from the cube geometry; do not edit.",
             "#pragma once", "#include <cstdint>", "namespace sph {",
             "__device__ const uint8_t kMcEdgeCorner[12][2] = {" +
             ", ".join("{%d, %d}" % e for e in EDGES) + "};",
             "__device__ const uint8_t kMcCornerOffset[8][3] = {" +
             ", ".join("{%d, %d, %d}" % c for c in CORNERS) + "};",
             "__device__ const uint16_t kMcEdgeFlags[256] = {"]
    for i in range(0, 256, 16):
        lines.append("    " + ", ".join(str(v) for v in ef[i:i + 16]) + ",")
    lines.append("};")
    lines.append("__device__ const int8_t kMcTriangles[256][16] = {")
    for row in tt:
        lines.append("    {" + ", ".join(str(v) for v in row) + "},")
    lines.append("};")
    lines.append("}  // namespace sph")
    open(os.path.join(here, "sph_mc_tables.h"), "w").write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
