"""Restart files (zj_restart_write / zj_restart_read): a run split by a
restart file equals the uninterrupted run bit for bit, time and iteration
resume, and files that do not fit the solver or are damaged are refused."""
import numpy as np
import pytest

from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu


def solver(P=3, n=8, **kw):
    mesh = M.tgv_mesh(n, seed=1)
    prm = make_params(poly_order=P, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      compat=False, viscous=True, Re=500.0, bcs=[(1, "slipwall")], **kw)
    return FRSolver(mesh, prm)


def test_split_run_is_identical(zjlib, tmp_path):
    a, b = solver(), solver()
    U0 = M.taylor_green(a.solution_point_coords())
    a.copyToDevice(U0)
    a.advance(1e-3, 20)
    b.copyToDevice(U0)
    b.advance(1e-3, 12)
    path = tmp_path / "r.zjr"
    b.write_restart(path)
    c = solver()
    c.read_restart(path)
    assert c.iteration == 12 and c.time == pytest.approx(12e-3, rel=0, abs=1e-15)
    c.advance(1e-3, 8)
    assert np.array_equal(c.copyToHost(), a.copyToHost())
    assert c.iteration == 20


def test_refuses_what_does_not_fit(zjlib, tmp_path):
    a = solver()
    a.copyToDevice(M.taylor_green(a.solution_point_coords()))
    path = tmp_path / "r.zjr"
    a.write_restart(path)
    for other in (solver(P=2), solver(n=6), solver(gamma=1.3)):
        with pytest.raises(L.ZJError) as e:
            other.read_restart(path)
        assert e.value.code == L.ERR_ARG
    raw = bytearray(path.read_bytes())
    raw[200] ^= 1
    bad = tmp_path / "bad.zjr"
    bad.write_bytes(bytes(raw))
    with pytest.raises(L.ZJError) as e:
        a.read_restart(bad)
    assert e.value.code == L.ERR_ARG and "checksum" in str(e.value)
    short = tmp_path / "short.zjr"
    short.write_bytes(bytes(raw[:20]))
    with pytest.raises(L.ZJError) as e:
        a.read_restart(short)
    assert e.value.code == L.ERR_IO
    with pytest.raises(L.ZJError) as e:
        a.read_restart(tmp_path / "missing.zjr")
    assert e.value.code == L.ERR_IO
