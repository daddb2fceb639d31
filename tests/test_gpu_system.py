"""The persistent linear-system seam (bsg_system, PetscLinearSystem's lifecycle) on the GPU.

The reference's own pressure-correction systems of three SIMPLE iterations on the 8^3
jittered-Voronoi cube (a new matrix once per outer iteration, then two non-orthogonal
corrector solves on the same matrix) are replayed through one persistent system.  The
preconditioner schedule (which solves rebuild the AMG hierarchy, which reuse a lagged one) must
equal the restatement of PetscLinearSystem's counters (petsc_linear_system.cpp:257-324,
446-470) fed with the same matrix changes and the device's iteration counts, and every
solution must agree with a direct solve.  Tolerance: rtol 1e-10 solves vs the direct solution
1e-8 relative L2.
"""
import numpy as np
import pytest

from helpers import Golden, ReferenceCounters, ref_system_groups, rel_l2
from oracle import fvm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def _pressure_sequence(g):
    seq = [s for grp in ref_system_groups(g) for s in grp["pressure"]]
    return seq + [seq[-1]]   # ten solves: the last one repeats an unchanged system


@pytest.mark.parametrize("interval", [8, 2])
def test_pressure_systems_follow_the_reference_rebuild_schedule(ctx, interval):
    import babelsim_b200 as bsg
    import scipy.sparse.linalg as spla
    g = Golden("voronoi8_config2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    geo = g.oracle_geometry()
    seq = _pressure_sequence(g)
    assert len(seq) == 10
    system = bsg.LinearSystem(m, 1)
    cfg = bsg.solver_config("cg", "hypre", 1e-15, 1e-10, 2000, rebuild_interval=interval)
    ref = ReferenceCounters(interval=interval)
    expected_setups = expected_reuses = 0
    previous = None
    for s in seq:
        changed = previous is None or any(not np.array_equal(s[k], previous[k]) for k in ("diag", "upper", "lower"))
        before = system.counters()
        x, res = system.solve(cfg, s["diag"], s["upper"], s["lower"], s["source"])
        after = system.counters()
        assert res[0].status == 0
        rebuilt = ref.solve(1 if changed else 0, res[0].iterations, res[0].status)
        expected_setups += int(rebuilt)
        expected_reuses += int(ref.lagged())
        assert after["preconditioner_setups"] - before["preconditioner_setups"] == int(rebuilt)
        assert after["matrix_value_updates"] - before["matrix_value_updates"] == int(changed)
        ldu = fvm.LDU(geo, False)
        ldu.diag, ldu.upper, ldu.lower, ldu.source = s["diag"], s["upper"], s["lower"], s["source"]
        exact = spla.spsolve(ldu.matrix().tocsc(), ldu.source)
        assert rel_l2(x, exact) < 1e-8
        previous = s
    k = system.counters()
    assert k["linear_solves"] == 10
    assert k["preconditioner_setups"] == expected_setups
    assert k["preconditioner_reuses"] == expected_reuses
    assert k["matrix_value_updates"] == 3 and k["rhs_only_solves"] == 7
    assert k["preconditioner_retries"] == 0
    assert k["true_residual_checks"] >= 10
    if interval == 2:
        assert expected_setups >= 2   # the lag expired at least once
    system.close()
    m.close()


def test_solve_ldu_reuses_its_system_across_calls(ctx):
    """bsg_solve_ldu keeps one persistent system per component count on the mesh: repeated calls
    give the same answers as a separate persistent system fed the same sequence."""
    import babelsim_b200 as bsg
    g = Golden("voronoi8_config2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    seq = _pressure_sequence(g)[:4]
    cfg = bsg.solver_config("cg", "hypre", 1e-15, 1e-10, 2000)
    fresh = bsg.LinearSystem(m, 1)
    for s in seq:
        x, res = bsg.solve_ldu(m, cfg, s["diag"], s["upper"], s["lower"], s["source"])
        y, _ = fresh.solve(cfg, s["diag"], s["upper"], s["lower"], s["source"])
        assert res[0].status == 0
        assert np.array_equal(x, y)  # the same lifecycle, the same kernels: bit for bit
    fresh.close()
    mom = ref_system_groups(g)[0]["momentum"]
    for _ in range(2):
        x, res = bsg.solve_ldu(m, bsg.solver_config("bcgs", "bjacobi", 1e-15, 1e-10, 2000), mom["diag"],
                               mom["upper"], mom["lower"], mom["source"].reshape(-1, 3))
        assert all(r.status == 0 for r in res)
    m.close()
