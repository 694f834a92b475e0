"""The C-ABI library: loads, exports every symbol include/zj_fr.h declares,
parses configs with the reference grammar, and reports errors as status codes
(never exits the process).  No compute call needs a GPU here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "zj_fr.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(zj_[a-z0-9_]+)\s*\(", txt)))


def test_exports_every_declared_symbol(zjlib):
    syms = declared_symbols()
    assert len(syms) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    for s in syms:
        getattr(zjlib, s)


def test_abi_version(zjlib):
    assert zjlib.zj_abi_version() == 1


def test_params_defaults_match_reference(zjlib):
    # SimParams defaults, include/common/types.hpp:130-172
    p = L.Params()
    zjlib.zj_params_default(C.byref(p))
    assert (p.gamma, p.Pr, p.Re, p.Mach, p.T_inf, p.p_inf, p.rho_inf, p.AoA) == \
        (1.4, 0.72, 1000.0, 0.5, 300.0, 101325.0, 1.225, 0.0)
    assert (p.poly_order, p.flux_type, p.riemann) == (3, L.FLUX_TYPES["HU"], L.RIEMANN["Roe"])
    assert (p.CFL, p.dt, p.t_final, p.max_iter, p.viscous) == (0.5, 0.0, 1.0, 100000, 1)
    assert (p.output_freq, p.restart_freq) == (100, 1000)
    assert p.case_name == b"simulation"


CONFIG = """# a test case
gamma       1.3         # ratio of specific heats
Pr          0.7
Re          2500
Mach        0.25
AoA         3.5
T_inf       288.0
p_inf       90000.0
rho_inf     1.1
poly_order  4
flux_type   SD
riemann     HLLC
CFL         0.3
dt          0.001
t_final     2.0
max_iter    77
viscous     false
output_freq 5
restart_freq 9
case_name   box
bc 1 farfield
bc 2 Slip_Wall
bc 3 outflow p_static 50000
bc 4 inflow p_total 120000 T_total 300 direction 0.0 1.0
bc 5 wall T_wall 500
bc 6 bogus
bc 3 outlet p_static 60000
unknown_key 12
compat off
precision mixed
"""


def test_config_grammar(zjlib):
    p = L.Params()
    zjlib.zj_params_default(C.byref(p))
    assert zjlib.zj_params_parse_string(CONFIG.encode(), C.byref(p)) == L.OK
    assert (p.gamma, p.Pr, p.Re, p.Mach, p.AoA, p.T_inf, p.p_inf, p.rho_inf) == \
        (1.3, 0.7, 2500.0, 0.25, 3.5, 288.0, 90000.0, 1.1)
    assert (p.poly_order, p.flux_type, p.riemann) == (4, 1, 2)
    assert (p.CFL, p.dt, p.t_final, p.max_iter, p.viscous) == (0.3, 0.001, 2.0, 77, 0)
    assert (p.output_freq, p.restart_freq, p.case_name) == (5, 9, b"box")
    assert (p.compat, p.precision) == (0, L.MIXED)
    bcs = {p.bc[i].tag: p.bc[i] for i in range(p.n_bc)}
    assert p.n_bc == 6
    assert bcs[1].type == L.BC_TYPES["farfield"]
    assert bcs[2].type == L.BC_TYPES["slipwall"]           # lower-cased type string
    assert bcs[3].type == L.BC_TYPES["outflow"] and bcs[3].p_static == 60000.0  # last wins
    assert bcs[4].type == L.BC_TYPES["inflow"]
    assert (bcs[4].p_total, bcs[4].T_total, bcs[4].dir_x, bcs[4].dir_y) == (120000.0, 300.0, 0.0, 1.0)
    assert bcs[5].type == L.BC_TYPES["wall"] and bcs[5].T_wall == 500.0
    assert bcs[6].type == L.BC_TYPES["slipwall"]            # unknown string -> slip wall


def test_config_file_missing(zjlib, tmp_path):
    p = L.Params()
    assert zjlib.zj_params_parse_file(str(tmp_path / "nope.txt").encode(), C.byref(p)) == L.ERR_IO
    f = tmp_path / "c.txt"
    f.write_text("poly_order 2\nflux_type GA\n")
    zjlib.zj_params_default(C.byref(p))
    assert zjlib.zj_params_parse_file(str(f).encode(), C.byref(p)) == L.OK
    assert (p.poly_order, p.flux_type) == (2, 3)


def _create(mesh, prm):
    return FRSolver(mesh, prm)


@pytest.mark.parametrize("P", [0, 6])
def test_bad_order_rejected(zjlib, P):
    with pytest.raises(L.ZJError) as e:
        _create(M.vortex_mesh(2), make_params(poly_order=P))
    assert e.value.code == L.ERR_ARG


def test_clockwise_mesh_rejected(zjlib):
    m = M.vortex_mesh(2)
    m.conn = m.conn[:, ::-1].copy()
    with pytest.raises(L.ZJError) as e:
        _create(m, make_params())
    assert e.value.code == L.ERR_ARG and "Jacobian" in str(e.value)


def test_bad_node_index_rejected(zjlib):
    m = M.vortex_mesh(2)
    m.conn[0, 0] = 10_000
    with pytest.raises(L.ZJError) as e:
        _create(m, make_params())
    assert e.value.code == L.ERR_ARG


def test_null_arguments(zjlib):
    h = C.c_void_p()
    assert zjlib.zj_solver_create(None, None, C.byref(h)) == L.ERR_ARG
    assert zjlib.zj_last_error(None)
    assert zjlib.zj_step(None, 0.1, 1) == L.ERR_ARG
    assert zjlib.zj_rhs(None, None, None) == L.ERR_ARG
    assert zjlib.zj_set_state_async(None, None) == L.ERR_ARG
    assert zjlib.zj_get_state_async(None, None) == L.ERR_ARG
    zjlib.zj_solver_destroy(None)


def test_empty_mesh_rejected(zjlib):
    """A mesh without elements (or without nodes) is refused with an argument
    error before any device work."""
    m = M.vortex_mesh(2)
    empty = M.QuadMesh(m.xy, m.conn[:0].copy(), m.bnd[:0].copy(), m.tag_names)
    with pytest.raises(L.ZJError) as e:
        _create(empty, make_params())
    assert e.value.code == L.ERR_ARG and "empty mesh" in str(e.value)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_no_device_reports_cuda_error(zjlib):
    with pytest.raises(L.ZJError) as e:
        _create(M.vortex_mesh(2), make_params())
    assert e.value.code == L.ERR_CUDA


def test_mixed_precision_needs_physics_mode(zjlib):
    """precision = mixed is the physics-mode form; compat mode (the
    reference's FP64 residual) refuses it before touching a device."""
    from zhijian_b200 import meshgen as M
    from zhijian_b200.solver import FRSolver, make_params
    with pytest.raises(L.ZJError) as e:
        FRSolver(M.vortex_mesh(4), make_params(compat=True, precision="mixed"))
    assert e.value.code == L.ERR_UNSUPPORTED


def test_precision_keys(zjlib):
    """precision fp64 | mixed (alias fp32) | split_bf16; split_bf16 is a
    physics-mode form like mixed and is refused in compat mode before any
    device work."""
    from zhijian_b200 import meshgen as M
    from zhijian_b200.solver import FRSolver, make_params
    for text, want in (("fp64", L.FP64), ("mixed", L.MIXED), ("fp32", L.MIXED), ("split_bf16", L.SPLIT_BF16)):
        p = L.Params()
        zjlib.zj_params_default(C.byref(p))
        assert zjlib.zj_params_parse_string(f"precision {text}\n".encode(), C.byref(p)) == L.OK
        assert p.precision == want
    with pytest.raises(L.ZJError) as e:
        FRSolver(M.vortex_mesh(4), make_params(compat=True, precision="split_bf16"))
    assert e.value.code == L.ERR_UNSUPPORTED
