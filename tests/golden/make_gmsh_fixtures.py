"""Gmsh fixtures and the reference reader's view of them.

    python tests/golden/make_gmsh_fixtures.py

writes small seeded ASCII meshes into tests/golden/gmsh/ (MSH v2.2 and v4.1:
Q1, Q2 and Q4 quads, serendipity quads, a mixed triangle/quad mesh, an
unnamed-group mesh, and four files the reader must refuse), then runs the
reference's GmshReader (oracle/_ref/ref_cpu "gmsh", compiled from the
reference sources by oracle/ref/Makefile) on each one and stores what it read
-- nodes, elements, faces with their boundary tags and types, boundary
groups -- or its failure, in tests/golden/ref_gmsh.npz.
"""
from __future__ import annotations

import math
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from zhijian_b200.meshgen import uniform01  # noqa: E402

OUT = os.path.join(HERE, "gmsh")
REF_CPU = os.path.join(ROOT, "oracle", "_ref", "ref_cpu")


def grid(nx, ny, order, x1=2.0, y1=1.5, jitter=0.1, seed=3, curve=0.0):
    """Nodes of an (order*nx+1) x (order*ny+1) lattice; interior nodes
    jittered; x bent by curve*sin(pi y/y1)."""
    mx, my = order * nx + 1, order * ny + 1
    r = uniform01(seed, 2 * mx * my).reshape(mx * my, 2)
    xy = []
    for j in range(my):
        for i in range(mx):
            x, y = x1 * i / (mx - 1), y1 * j / (my - 1)
            k = j * mx + i
            if 0 < i < mx - 1 and 0 < j < my - 1:
                x += (2 * r[k, 0] - 1) * jitter * x1 / (mx - 1)
                y += (2 * r[k, 1] - 1) * jitter * y1 / (my - 1)
            x += curve * math.sin(math.pi * y / y1)
            xy.append((x, y))
    return xy, mx, my


def quad_cells(nx, ny, order, mx):
    """Gmsh node order of each cell (0-based lattice indices): corners CCW,
    then the edge and interior nodes of the order."""
    cells = []
    for cj in range(ny):
        for ci in range(nx):
            i0, j0 = order * ci, order * cj
            n = lambda a, b: (j0 + b) * mx + (i0 + a)
            o = order
            c = [n(0, 0), n(o, 0), n(o, o), n(0, o)]
            if order == 2:
                c += [n(1, 0), n(2, 1), n(1, 2), n(0, 1), n(1, 1)]
            elif order == 4:
                # corners, edges (3 each, CCW), then the interior 3x3 block
                c += [n(1, 0), n(2, 0), n(3, 0), n(4, 1), n(4, 2), n(4, 3),
                      n(3, 4), n(2, 4), n(1, 4), n(0, 3), n(0, 2), n(0, 1)]
                c += [n(1, 1), n(3, 1), n(3, 3), n(1, 3), n(2, 1), n(3, 2), n(2, 3), n(1, 2), n(2, 2)]
            cells.append(c)
    return cells


def sides(nx, ny, order, mx, my):
    """Boundary segments of the lattice per side (bottom, right, top, left),
    each as its node list (end vertices first for order 2)."""
    o = order
    segs = {0: [], 1: [], 2: [], 3: []}
    for ci in range(nx):
        a, b = o * ci, o * (ci + 1)
        segs[0].append([a, b] + ([a + 1] if o == 2 else []))
        top = (my - 1) * mx
        segs[2].append([top + b, top + a] + ([top + a + 1] if o == 2 else []))
    for cj in range(ny):
        a, b = o * cj, o * (cj + 1)
        segs[1].append([a * mx + mx - 1, b * mx + mx - 1] + ([(a + 1) * mx + mx - 1] if o == 2 else []))
        segs[3].append([b * mx, a * mx] + ([(a + 1) * mx] if o == 2 else []))
    return segs


NAMES = {1: "wall", 2: "outlet", 3: "SlipWall", 4: "farfield"}


def write_v22(path, xy, cells, ctype, segs, ltype, names=NAMES, tag_base=10, extra=()):
    tags = [tag_base + 3 * k for k in range(len(xy))]
    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat"]
    if names:
        lines += ["$PhysicalNames", str(len(names) + 1)]
        lines += [f'1 {t} "{n}"' for t, n in names.items()]
        lines += ['2 100 "fluid"', "$EndPhysicalNames"]
    lines += ["$Nodes", str(len(xy))]
    lines += [f"{tags[k]} {x:.17g} {y:.17g} 0" for k, (x, y) in enumerate(xy)]
    lines += ["$EndNodes"]
    els = [f"15 2 0 1 {tags[0]}"]    # a point element, skipped
    for side, ss in segs.items():
        for s in ss:
            els.append(f"{ltype} 2 {side + 1} {side + 11} " + " ".join(str(tags[v]) for v in s))
    for c in cells:
        els.append(f"{ctype} 2 100 1 " + " ".join(str(tags[v]) for v in c))
    els += list(extra)
    lines += ["$Elements", str(len(els))]
    lines += [f"{k + 1} {e}" for k, e in enumerate(els)]
    lines += ["$EndElements", "$Comments", "skipped section", "$EndComments"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_v41(path, xy, cells, ctype, segs, ltype, names=NAMES, file_type=0, tri=()):
    tags = [5 + 2 * k for k in range(len(xy))]
    lines = ["$MeshFormat", f"4.1 {file_type} 8", "$EndMeshFormat"]
    lines += ["$PhysicalNames", str(len(names) + 1)]
    lines += [f'1 {t} "{n}"' for t, n in names.items()] + ['2 100 "fluid"', "$EndPhysicalNames"]
    # entities: 0 points, 4 curves (curve c+21 -> physical c+1), 1 surface
    lines += ["$Entities", "0 4 1 0"]
    for c in range(4):
        lines.append(f"{c + 21} 0 0 0 2 1.5 0 1 {c + 1} 0")
    lines += ["1 0 0 0 2 1.5 0 1 100 0", "$EndEntities"]
    lines += ["$Nodes", f"1 {len(xy)} {min(tags)} {max(tags)}", f"2 1 0 {len(xy)}"]
    lines += [str(t) for t in tags]
    lines += [f"{x:.17g} {y:.17g} 0" for x, y in xy]
    lines += ["$EndNodes"]
    blocks = []
    eid = 1
    for side, ss in segs.items():
        b = [f"1 {side + 21} {ltype} {len(ss)}"]
        for s in ss:
            b.append(f"{eid} " + " ".join(str(tags[v]) for v in s)); eid += 1
        blocks.append(b)
    b = [f"2 1 {ctype} {len(cells)}"]
    for c in cells:
        b.append(f"{eid} " + " ".join(str(tags[v]) for v in c)); eid += 1
    blocks.append(b)
    if tri:
        b = [f"2 1 2 {len(tri)}"]
        for t in tri:
            b.append(f"{eid} " + " ".join(str(tags[v]) for v in t)); eid += 1
        blocks.append(b)
    n_el = sum(len(b) - 1 for b in blocks)
    lines += ["$Elements", f"{len(blocks)} {n_el} 1 {eid - 1}"]
    for b in blocks:
        lines += b
    lines += ["$EndElements"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def fixtures():
    os.makedirs(OUT, exist_ok=True)
    made = {}
    xy, mx, my = grid(4, 3, 1)
    cells, segs = quad_cells(4, 3, 1, mx), sides(4, 3, 1, mx, my)
    write_v22(os.path.join(OUT, "quad_v22.msh"), xy, cells, 3, segs, 1)
    write_v41(os.path.join(OUT, "quad_v41.msh"), xy, cells, 3, segs, 1)
    made["quad_v22"] = made["quad_v41"] = True
    # no physical names: groups "BC_<tag>", inferred as walls
    write_v22(os.path.join(OUT, "nophys_v22.msh"), xy, cells, 3, segs, 1, names=None)
    made["nophys_v22"] = True
    # Q2 (9-node) with curved sides, v4.1; serendipity (8-node) with 3-node lines, v2.2
    xy2, mx2, my2 = grid(2, 2, 2, curve=0.08, seed=5)
    c2, s2 = quad_cells(2, 2, 2, mx2), sides(2, 2, 2, mx2, my2)
    write_v41(os.path.join(OUT, "quad2_v41.msh"), xy2, c2, 10, s2, 8)
    write_v22(os.path.join(OUT, "serendipity_v22.msh"), xy2, [c[:8] for c in c2], 16, s2, 8)
    made["quad2_v41"] = made["serendipity_v22"] = True
    # Q4 (25-node), one layer of 2 cells, v2.2 (end vertices of each side line)
    xy4, mx4, my4 = grid(2, 1, 4, curve=0.05, seed=6)
    c4 = quad_cells(2, 1, 4, mx4)
    s4 = {k: [s[:2] for s in v] for k, v in sides(2, 1, 4, mx4, my4).items()}
    write_v22(os.path.join(OUT, "quad4_v22.msh"), xy4, c4, 37, s4, 1)
    made["quad4_v22"] = True
    # mixed: the right column of quads split into two triangles each
    keep = [c for k, c in enumerate(cells) if k % 4 != 3]
    tris = []
    for k, c in enumerate(cells):
        if k % 4 == 3:
            tris += [[c[0], c[1], c[2]], [c[0], c[2], c[3]]]
    write_v41(os.path.join(OUT, "triquad_v41.msh"), xy, keep, 3, segs, 1, tri=tris)
    made["triquad_v41"] = True
    # failures
    write_v41(os.path.join(OUT, "binary_v41.msh"), xy, cells, 3, segs, 1, file_type=1)
    write_v22(os.path.join(OUT, "unknown_node_v22.msh"), xy, cells, 3, segs, 1,
              extra=["3 2 100 1 1 2 3 99999"])
    with open(os.path.join(OUT, "no2d_v22.msh"), "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n2\n1 0 0 0\n2 1 0 0\n$EndNodes\n"
                "$Elements\n2\n1 15 1 1 1\n2 1 1 1 1 2\n$EndElements\n")
    with open(os.path.join(OUT, "tet_v22.msh"), "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n4\n1 0 0 0\n2 1 0 0\n3 0 1 0\n"
                "4 0 0 1\n$EndNodes\n$Elements\n1\n1 4 0 1 2 3 4\n$EndElements\n")
    for k in ("binary_v41", "unknown_node_v22", "no2d_v22", "tet_v22"):
        made[k] = False
    return made


def read_dump(path):
    b = open(path, "rb").read()
    o = 0

    def get(fmt):
        nonlocal o
        v = struct.unpack_from(fmt, b, o)
        o += struct.calcsize(fmt)
        return v
    nn, = get("<q")
    xy = np.array(get(f"<{2 * nn}d")).reshape(nn, 2)
    ne, = get("<q")
    et, eo, conn, off = [], [], [], [0]
    for _ in range(ne):
        t, order, k = get("<3i")
        et.append(t); eo.append(order)
        conn += list(get(f"<{k}q"))
        off.append(len(conn))
    nf, = get("<q")
    faces = np.array([get("<6i") for _ in range(nf)], dtype=np.int32).reshape(nf, 6)
    ng, = get("<i")
    groups = np.array([get("<2i") for _ in range(ng)], dtype=np.int32).reshape(ng, 2)
    return dict(xy=xy, elem_type=np.array(et, np.int32), elem_order=np.array(eo, np.int32),
                offsets=np.array(off, np.int64), conn=np.array(conn, np.int64), faces=faces,
                groups=groups)


def main():
    made = fixtures()
    if not os.path.exists(REF_CPU):
        print("reference reader not built (oracle/_ref/ref_cpu): fixtures only")
        return
    out = {}
    for name, ok in made.items():
        dump = os.path.join("/tmp", f"ref_gmsh_{name}.bin")
        r = subprocess.run([REF_CPU, "gmsh", os.path.join(OUT, name + ".msh"), dump],
                           capture_output=True, text=True)
        if ok:
            assert r.returncode == 0, (name, r.stderr)
            for k, v in read_dump(dump).items():
                out[f"{name}/{k}"] = v
        else:
            assert r.returncode != 0, name
            out[f"{name}/error"] = np.array(r.stderr.strip().splitlines()[0])
    np.savez_compressed(os.path.join(HERE, "ref_gmsh.npz"), **out)
    print("wrote", len(made), "fixtures and", os.path.join(HERE, "ref_gmsh.npz"))


if __name__ == "__main__":
    main()
