"""Mixed precision against the FP64 path, the direct solve and the reference: FP32
inner PCG and FP32 AMG V-cycles inside FP64 iterative refinement (precision 1),
FP64 flexible PCG with FP32 V-cycles (precision 2), and FP32 inner Jacobi BiCGStab
inside FP64 refinement for the momentum systems (precision 1 on the momentum solver).

Tolerances: the refined solve meets the same FP64 true-residual contract as
the FP64 path, so solutions agree with a direct solve to 1e-8 (rtol 1e-12) and
converged SIMPLE fields with the reference's to 1e-8 after the reference's own number of
outer iterations (outer tolerance 1e-6); the bound asked of the mixed path is 1e-6
relative L2 of the FP64 result.
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


@pytest.mark.parametrize("components", [1, 3])
@pytest.mark.parametrize("rtol", [1e-12, 1e-8])
def test_refined_bicgstab_momentum_system(ctx, rtol, components):
    """The reference's non-symmetric momentum system (8^3 jittered-Voronoi cube, linearUpwind),
    all three components together or the x component alone, through the C ABI."""
    import babelsim_b200 as bsg
    from test_gpu_gmres import _direct
    g = Golden("voronoi8_config2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    mom = ref_system_groups(g)[0]["momentum"]
    vector = components == 3
    s = dict(mom) if vector else dict(mom, source=mom["source"].reshape(-1, 3)[:, 0].copy())
    exact, ldu = _direct(g.oracle_geometry(), s, vector)
    b = s["source"].reshape(-1, 3) if vector else s["source"]
    x, res = bsg.solve_ldu(m, bsg.solver_config("bcgs", "bjacobi", 1e-30, rtol, 3000, precision=1), s["diag"],
                           s["upper"], s["lower"], b)
    x64, res64 = bsg.solve_ldu(m, bsg.solver_config("bcgs", "bjacobi", 1e-30, rtol, 3000), s["diag"], s["upper"],
                               s["lower"], b)
    bb = b.reshape(len(b), -1)
    xx = x.reshape(len(b), -1)
    for c in range(components):
        col = bb[:, c].copy()
        # (the first outer iteration's y and z sources are zero: nothing to iterate there)
        assert res[c].status == 0 and (res[c].iterations > 0 or not np.any(col))
        # the FP64 true-residual contract of the FP64 path (zero initial guess: ||r0|| = ||b||)
        r = col - ldu.apply(xx[:, c].copy())
        assert np.linalg.norm(r) <= rtol * np.linalg.norm(col) * 1.0000001
        assert res[c].final_residual <= rtol * np.linalg.norm(col) * 1.0000001
    assert rel_l2(x, exact) < max(1e-8, 1e4 * rtol)
    assert rel_l2(x, x64) < max(1e-8, 1e4 * rtol)
    m.close()


def _mixed_simple(bsg, g, m, precision, momentum_precision=0):
    s = g.settings()
    sol = g.meta["solution"]
    sim = bsg.Simple(m, s.rho, s.mu, s.alpha_u, s.alpha_p, s.non_orthogonal_corrections, s.mass_tolerance,
                     s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
                     bsg.options(**s.momentum), bsg.options(**s.pressure),
                     bsg.solver_config("bcgs", "bjacobi", sol["equation.momentum.absoluteTolerance"],
                                       sol["equation.momentum.relativeTolerance"], 2000,
                                       precision=momentum_precision),
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


@pytest.mark.parametrize("name", ["warped5_corrected", "cavity64_config1", "voronoi8_config2"])
def test_mixed_momentum_simple_converges_to_reference(ctx, name):
    """FP32 inner iterations for both the momentum and the pressure solves."""
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    target = int(g["conv_info"][1])
    r, U, p = fields_at_reference_count(lambda: _mixed_simple(bsg, g, m, 1, momentum_precision=1), m.n_cells,
                                        target)
    assert r.converged
    assert abs(r.iterations - target) <= 2
    assert rel_l2(U, g["U_conv"]) < 1e-8
    assert rel_l2(p, g["p_conv"]) < 1e-8
    m.close()
