"""The oracle is pinned to the reference's own code: operators, faces,
normals and metric terms bit for bit against the reference's basis.cpp,
mesh.cpp and initGeometry (fixtures written by tests/golden/make_golden.py from
oracle/_ref/ref_cpu), and the residual against the reference's CUDA build
(ref_gpu_residuals.npz, written on a B200 by the same script)."""
import os

import numpy as np
import pytest

from tests import _util as U_
from tests.golden import make_golden as G

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
def test_operators_bitwise(oracle_mod, P):
    ref = np.load(os.path.join(GOLD, "ref_operators.npz"))
    orc = oracle_mod.Oracle(G.mixed_mesh(), P)
    mine = orc.operators()
    for k in ("pts", "D1", "diff_xi", "diff_eta", "interp", "corr"):
        assert np.array_equal(ref[f"P{P}_{k}"], mine[k]), k


@pytest.mark.parametrize("name,P", [("mixed", 3), ("mixed", 5), ("tgv12", 3)])
def test_mesh_geometry_bitwise(oracle_mod, name, P):
    ref = np.load(os.path.join(GOLD, "ref_geometry.npz"))
    if name == "mixed":
        mesh, tags = G.mixed_mesh(), G.mixed_tags(0.9e5)
    else:
        from zhijian_b200 import meshgen as M
        mesh, tags = M.tgv_mesh(12, seed=1), None
    orc = oracle_mod.Oracle(mesh, P, tags=tags)
    f = orc.faces()
    key = f"{name}_P{P}"
    for a, b in (("le", "left_elem"), ("ll", "left_local"), ("re", "right_elem"),
                 ("rl", "right_local"), ("bct", "bc_type"), ("tag", "bc_tag")):
        assert np.array_equal(ref[f"{key}_face_{a}"], f[b]), a
    assert np.array_equal(ref[f"{key}_face_nx"], f["normals"][:, 0])
    assert np.array_equal(ref[f"{key}_face_ny"], f["normals"][:, 1])
    J, Ji = orc.geometry()
    assert np.array_equal(ref[f"{key}_J"], J)
    assert np.array_equal(ref[f"{key}_Jinv"], Ji)
    assert np.array_equal(ref[f"{key}_spxy"], orc.sp_coords())


def _gpu_goldens():
    p = os.path.join(GOLD, "ref_gpu_residuals.npz")
    return np.load(p) if os.path.exists(p) else None


@pytest.mark.parametrize("name", sorted(G.case_defs()))
def test_oracle_residual_vs_reference_gpu(oracle_mod, name):
    gold = _gpu_goldens()
    assert gold is not None, "ref_gpu_residuals.npz missing: run make_golden.py gpu on a B200"
    c = G.case_defs()[name]
    rho, p, mach, aoa = c["prm"]
    orc = oracle_mod.Oracle(c["mesh"], c["P"], G.GAMMA, rho, p, mach, aoa, tags=c["tags"])
    U = gold[f"{name}_U"]
    assert np.array_equal(U, G.make_state(c, orc.sp_coords()))
    R = orc.rhs(U)
    Rref = gold[f"{name}_R"]
    s = U_.euler_flux_scale(U, orc.geometry()[1])
    # the reference CUDA build contracts to FMA, the oracle rounds every op
    assert U_.rel_err(R, Rref, s) <= 1e-13
    if f"{name}_Ustep" in gold:
        Us, Rs = orc.step(U, c["dt"], c["nsteps"])
        ss = U_.euler_flux_scale(gold[f"{name}_Ustep"])
        assert U_.rel_err(Us, gold[f"{name}_Ustep"], ss) <= 1e-12
        norm = orc_norm = float(np.sqrt(np.sum(Rs * Rs)))
        assert abs(orc_norm - gold[f"{name}_norm"][0]) <= 1e-11 * max(norm, 1.0)
