"""The Gmsh reader (zj_gmsh_read) against the reference's GmshReader
(src/mesh/gmsh_reader.cpp) on the fixtures of tests/golden/gmsh/: nodes,
elements, boundary groups with their inferred types, and every boundary
face's tag and type must be identical (tests/golden/ref_gmsh.npz, made by
tests/golden/make_gmsh_fixtures.py with the reference reader compiled from
its sources); the files the reference refuses are refused with its message.
No device is needed."""
import os

import numpy as np
import pytest

from zhijian_b200 import _lib as L
from zhijian_b200.gmsh import read_gmsh

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
REF = np.load(os.path.join(GOLD, "ref_gmsh.npz"))
GOOD = sorted({k.split("/")[0] for k in REF.files if not k.endswith("/error")})
BAD = sorted({k.split("/")[0] for k in REF.files if k.endswith("/error")})


def fixture(name):
    return os.path.join(GOLD, "gmsh", name + ".msh")


@pytest.mark.parametrize("name", GOOD)
def test_reader_matches_reference(zjlib, name):
    g = read_gmsh(fixture(name))
    ref = {k.split("/")[1]: REF[k] for k in REF.files if k.startswith(name + "/")}
    assert np.array_equal(g.xy, ref["xy"])
    assert np.array_equal(g.elem_type, ref["elem_type"])
    assert np.array_equal(g.elem_order, ref["elem_order"])
    assert np.array_equal(g.offsets, ref["offsets"])
    assert np.array_equal(g.conn, ref["conn"])
    assert [(t, ty) for t, ty, _ in g.groups] == [tuple(r) for r in ref["groups"]]
    # boundary faces: the tag of the last edge with the face's vertex pair
    tags = {}
    for v0, v1, t in g.bnd:
        tags[(min(v0, v1), max(v0, v1))] = int(t)
    types = {t: ty for t, ty, _ in g.groups}
    n_checked = 0
    for le, lf, re, rf, bct, tag in ref["faces"]:
        if re >= 0:
            continue
        el = g.element(le)
        nv = 3 if g.elem_type[le] == 0 else 4
        a, b = int(el[lf % nv]), int(el[(lf + 1) % nv])
        mine = tags.get((min(a, b), max(a, b)))
        if tag > 0:
            assert mine == tag
            assert types[mine] == bct
            n_checked += 1
        else:
            assert mine is None
    assert n_checked > 0


@pytest.mark.parametrize("name", BAD)
def test_reader_refuses_what_the_reference_refuses(zjlib, name):
    with pytest.raises(L.ZJError) as e:
        read_gmsh(fixture(name))
    assert e.value.code == L.ERR_ARG
    assert str(REF[name + "/error"]) in str(e.value)


def test_missing_file(zjlib):
    with pytest.raises(L.ZJError) as e:
        read_gmsh(fixture("does_not_exist"))
    assert e.value.code == L.ERR_IO


def test_group_names_and_inferred_types(zjlib):
    g = read_gmsh(fixture("quad_v41"))
    assert g.groups == [
        (1, L.BC_TYPES["wall"], "wall"), (2, L.BC_TYPES["outflow"], "outlet"),
        (3, L.BC_TYPES["slipwall"], "SlipWall"), (4, L.BC_TYPES["farfield"], "farfield")]
    assert [n for _, _, n in read_gmsh(fixture("nophys_v22")).groups] == ["BC_1", "BC_2", "BC_3", "BC_4"]
    # the serendipity quads gained a centre node each
    s = read_gmsh(fixture("serendipity_v22"))
    q = read_gmsh(fixture("quad2_v41"))
    assert s.xy.shape[0] == q.xy.shape[0] + 4
    assert set(s.elem_order.tolist()) == {2}
