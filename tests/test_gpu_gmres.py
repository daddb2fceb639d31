"""GMRES(30) and FGMRES(30) on the device (kspType gmres / fgmres, KSPGMRES / KSPFGMRES in
src/backend/petsc_linear_system.cpp:43-50), through the C ABI.

Systems: the reference's own non-symmetric momentum matrix (linearUpwind convection on the
8^3 jittered-Voronoi cube, first outer iteration) and its pressure-correction system.  Each
solve must meet the reference's acceptance contract (true residual <= rtol * max(||r0||,
||b||)) and agree with a direct solve to 1e-8 relative L2 at rtol 1e-12.
"""
import numpy as np
import pytest

from helpers import Golden, fields_at_reference_count, ref_system_groups, rel_l2
from oracle import fvm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def _direct(geo, s, vector):
    import scipy.sparse.linalg as spla
    ldu = fvm.LDU(geo, vector)
    ldu.diag, ldu.upper, ldu.lower = s["diag"], s["upper"], s["lower"]
    lu = spla.splu(ldu.matrix().tocsc())
    b = s["source"].reshape(-1, 3) if vector else s["source"]
    if vector:
        return np.stack([lu.solve(b[:, c].copy()) for c in range(3)], 1), ldu
    return lu.solve(b.copy()), ldu


@pytest.mark.parametrize("ksp", ["gmres", "fgmres"])
@pytest.mark.parametrize("pc", ["jacobi", "none"])
def test_scalar_nonsymmetric_system(ctx, ksp, pc):
    """The x component of the momentum system as a scalar, non-symmetric system."""
    import babelsim_b200 as bsg
    g = Golden("voronoi8_config2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    mom = ref_system_groups(g)[0]["momentum"]
    s = dict(diag=mom["diag"], upper=mom["upper"], lower=mom["lower"], source=mom["source"].reshape(-1, 3)[:, 0].copy())
    exact, ldu = _direct(g.oracle_geometry(), s, False)
    x, res = bsg.solve_ldu(m, bsg.solver_config(ksp, pc, 1e-30, 1e-12, 3000), s["diag"], s["upper"], s["lower"],
                           s["source"])
    assert res[0].status == 0 and res[0].iterations > 0
    r = s["source"] - ldu.apply(x)
    assert np.linalg.norm(r) <= 1e-12 * np.linalg.norm(s["source"]) * 1.0000001
    assert res[0].final_residual <= 1e-12 * np.linalg.norm(s["source"]) * 1.0000001
    assert rel_l2(x, exact) < 1e-8
    m.close()


@pytest.mark.parametrize("ksp", ["gmres", "fgmres"])
def test_vector_system_three_components(ctx, ksp):
    import babelsim_b200 as bsg
    g = Golden("voronoi8_config2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    mom = ref_system_groups(g)[0]["momentum"]
    exact, _ = _direct(g.oracle_geometry(), mom, True)
    x, res = bsg.solve_ldu(m, bsg.solver_config(ksp, "bjacobi", 1e-30, 1e-12, 3000), mom["diag"], mom["upper"],
                           mom["lower"], mom["source"].reshape(-1, 3))
    assert all(r.status == 0 for r in res)
    assert rel_l2(x, exact) < 1e-8
    m.close()


@pytest.mark.parametrize("ksp", ["gmres", "fgmres"])
def test_pressure_system_with_amg(ctx, ksp):
    """GMRES / FGMRES right-preconditioned by the device AMG V-cycle (pcType hypre)."""
    import babelsim_b200 as bsg
    g = Golden("voronoi8_config2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sysp = ref_system_groups(g)[0]["pressure"][0]
    exact, _ = _direct(g.oracle_geometry(), sysp, False)
    x, res = bsg.solve_ldu(m, bsg.solver_config(ksp, "hypre", 1e-30, 1e-12, 3000), sysp["diag"], sysp["upper"],
                           sysp["lower"], sysp["source"])
    assert res[0].status == 0
    assert res[0].iterations < 200
    assert rel_l2(x, exact) < 1e-8
    m.close()


def test_simple_with_gmres_momentum_reaches_reference_fields(ctx):
    """A SIMPLE run whose momentum equation is configured with kspType gmres converges to the
    reference's fields (the converged state does not depend on the Krylov method)."""
    import babelsim_b200 as bsg
    g = Golden("cavity12_upwind")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    s = g.settings()
    sol = g.meta["solution"]

    def make():
        sim = bsg.Simple(m, s.rho, s.mu, s.alpha_u, s.alpha_p, s.non_orthogonal_corrections, s.mass_tolerance,
                         s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
                         bsg.options(**s.momentum), bsg.options(**s.pressure),
                         bsg.solver_config("gmres", "bjacobi", sol["equation.momentum.absoluteTolerance"],
                                           sol["equation.momentum.relativeTolerance"], 2000),
                         bsg.solver_config("cg", "hypre", sol["equation.pressureCorrection.absoluteTolerance"],
                                           sol["equation.pressureCorrection.relativeTolerance"], 20000))
        for p, (t, v) in enumerate(g.meta["U_bcs"]):
            sim.set_boundary("U", p, t, v)
        for p, (t, v) in enumerate(g.meta["p_bcs"]):
            sim.set_boundary("p", p, t, v)
        return sim
    target = int(g["conv_info"][1])
    r, U, p = fields_at_reference_count(make, m.n_cells, target)
    assert r.converged and abs(r.iterations - target) <= 2
    assert rel_l2(U, g["U_conv"]) < 1e-8
    assert rel_l2(p, g["p_conv"]) < 1e-8
    m.close()
