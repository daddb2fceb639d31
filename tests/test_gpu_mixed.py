"""Mixed precision against the FP64 path, the direct solve and the reference: FP32
inner PCG and FP32 AMG V-cycles inside FP64 iterative refinement (precision 1),
and FP64 flexible PCG with FP32 V-cycles (precision 2).

Tolerances: the refined solve meets the same FP64 true-residual contract as
the FP64 path, so solutions agree with a direct solve to 1e-8 (rtol 1e-12) and
converged SIMPLE fields with the reference's to 1e-8 after the reference's own number of
outer iterations (outer tolerance 1e-6); the
north star's bound for the mixed path is 1e-6 relative L2 of the FP64 result.
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


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("rtol", [1e-12, 1e-8])
def test_refined_pressure_solve(ctx, rtol, precision):
    import babelsim_b200 as bsg
    import scipy.sparse.linalg as spla
    g = Golden("cavity64_config1")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sysp = ref_system_groups(g)[0]["pressure"][0]
    geo = g.oracle_geometry()
    ldu = fvm.LDU(geo, False)
    ldu.diag, ldu.upper, ldu.lower, ldu.source = sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"]
    exact = spla.spsolve(ldu.matrix().tocsc(), ldu.source)
    cfg = bsg.solver_config("cg", "hypre", 1e-30, rtol, 20000, precision=precision)
    x, res = bsg.solve_ldu(m, cfg, sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"])
    assert res[0].status == 0
    # FP64 true residual contract, whatever the inner precision
    r = ldu.source - ldu.apply(x)
    assert np.linalg.norm(r) <= rtol * np.linalg.norm(sysp["source"]) * 1.0000001
    assert rel_l2(x, exact) < max(1e-8, 1e4 * rtol)
    m.close()


def _mixed_simple(bsg, g, m, precision):
    s = g.settings()
    sol = g.meta["solution"]
    sim = bsg.Simple(m, s.rho, s.mu, s.alpha_u, s.alpha_p, s.non_orthogonal_corrections, s.mass_tolerance,
                     s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
                     bsg.options(**s.momentum), bsg.options(**s.pressure),
                     bsg.solver_config("bcgs", "bjacobi", sol["equation.momentum.absoluteTolerance"],
                                       sol["equation.momentum.relativeTolerance"], 2000),
                     bsg.solver_config("cg", "hypre", sol["equation.pressureCorrection.absoluteTolerance"],
                                       sol["equation.pressureCorrection.relativeTolerance"], 20000,
                                       precision=precision))
    for p, (t, v) in enumerate(g.meta["U_bcs"]):
        sim.set_boundary("U", p, t, v)
    for p, (t, v) in enumerate(g.meta["p_bcs"]):
        sim.set_boundary("p", p, t, v)
    return sim


@pytest.mark.parametrize("precision", [1, 2])
@pytest.mark.parametrize("name", ["warped5_corrected", "cavity64_config1", "voronoi8_config2"])
def test_mixed_simple_converges_to_reference(ctx, name, precision):
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    target = int(g["conv_info"][1])
    r, U, p = fields_at_reference_count(lambda: _mixed_simple(bsg, g, m, precision), m.n_cells, target)
    assert r.converged
    assert abs(r.iterations - target) <= 2
    assert rel_l2(U, g["U_conv"]) < 1e-8
    assert rel_l2(p, g["p_conv"]) < 1e-8
    m.close()
