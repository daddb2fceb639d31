"""Block-diagonal batching (bsg_simple_set_segments): several independent SIMPLE cases
concatenated into one mesh, advanced by one set of kernel launches, their pressure systems
solved in one persistent launch per attempt.

Each case of the batch must give what it gives alone.  The batch runs the same kernels on the
same rows, except that each case's persistent pressure solve runs on fewer CTAs than the whole
grid, which changes the order of its dot-product sums: after a fixed number of outer iterations
the fields agree with the solo run's to 1e-9 relative L2 (rounding only); run to convergence,
each case converges within one outer iteration of its solo count and its converged U and p
agree to 1e-7.  The 8^3 Voronoi case also still meets the reference's converged fields.
"""
import numpy as np
import pytest

from helpers import Golden, rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


LID = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", None)] + [("fixedValue", (0.0, 0.0, 0.0))] * 2


def _cases():
    v = Golden("voronoi8_config2").poly
    w = Golden("warped5_corrected").poly
    # (mesh, lid speed, dynamic viscosity): uneven sizes and settings
    return [(v, 1.0, 1e-3), (w, 1.0, 1e-2), (v, 2.0, 4e-3)]


def _make(bsg, mesh, mu):
    opts = bsg.options("linear", "leastSquares", "linearUpwind", "corrected")
    return bsg.Simple(mesh, 1.0, mu, 0.7, 0.3, 2, 1e-6, 1e-6, 1e-6, 1e-6, opts, opts,
                      bsg.solver_config("bcgs", "bjacobi", 1e-15, 1e-10, 2000),
                      bsg.solver_config("cg", "hypre", 1e-15, 1e-10, 5000))


def _set_bcs(sim, patch0, lid):
    for p, (t, v) in enumerate(LID):
        sim.set_boundary("U", patch0 + p, t, (lid, 0.0, 0.0) if v is None else v)
        sim.set_boundary("p", patch0 + p, "zeroGradient")


def _solo(bsg, ctx, poly, lid, mu, iterations):
    m = bsg.Mesh.from_polyhedral(ctx, poly)
    sim = _make(bsg, m, mu)
    _set_bcs(sim, 0, lid)
    n = m.n_cells
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    r = sim.iterate(iterations)
    U, p, _ = sim.fields()
    sim.close()
    m.close()
    return r, U, p


def _batch(bsg, ctx, cases):
    from babelsim_b200 import meshgen
    poly, cells, patches = meshgen.concatenate([c[0] for c in cases])
    m = bsg.Mesh.from_polyhedral(ctx, poly)
    sim = _make(bsg, m, cases[0][2])
    sim.set_segments(cells, [c[2] for c in cases])
    for k, c in enumerate(cases):
        _set_bcs(sim, int(patches[k]), c[1])
    sim.set_fields(np.zeros((m.n_cells, 3)), np.zeros(m.n_cells))
    return m, sim, cells


def test_batch_equals_solo_after_fixed_iterations(ctx):
    import babelsim_b200 as bsg
    cases = _cases()
    m, sim, cells = _batch(bsg, ctx, cases)
    r = sim.iterate(12)
    assert r.iterations == 12 and r.status == 1
    U, p, _ = sim.fields()
    for k, (poly, lid, mu) in enumerate(cases):
        _, Us, ps = _solo(bsg, ctx, poly, lid, mu, 12)
        a, b = cells[k], cells[k + 1]
        assert rel_l2(U[a:b], Us) < 1e-9, k
        assert rel_l2(p[a:b], ps) < 1e-9, k
        assert sim.segment_report(k).iterations == 12
    sim.close()
    m.close()


def test_batch_converges_each_case_as_alone(ctx):
    import babelsim_b200 as bsg
    cases = _cases()
    m, sim, cells = _batch(bsg, ctx, cases)
    r = sim.iterate(3000)
    assert r.converged and r.status == 0
    U, p, _ = sim.fields()
    for k, (poly, lid, mu) in enumerate(cases):
        rs, Us, ps = _solo(bsg, ctx, poly, lid, mu, 3000)
        seg = sim.segment_report(k)
        assert seg.converged and rs.converged
        assert abs(seg.iterations - rs.iterations) <= 1, (k, seg.iterations, rs.iterations)
        a, b = cells[k], cells[k + 1]
        assert rel_l2(U[a:b], Us) < 1e-7, k
        assert rel_l2(p[a:b], ps) < 1e-7, k
    # the first case is the reference's own 8^3 Voronoi fixture case (same mesh and settings)
    g = Golden("voronoi8_config2")
    a, b = cells[0], cells[1]
    assert abs(sim.segment_report(0).iterations - int(g["conv_info"][1])) <= 2
    assert rel_l2(U[a:b], g["U_conv"]) < 1e-6
    assert rel_l2(p[a:b], g["p_conv"]) < 1e-6
    sim.close()
    m.close()


def test_segments_must_be_independent(ctx):
    import babelsim_b200 as bsg
    poly = Golden("voronoi8_config2").poly
    m = bsg.Mesh.from_polyhedral(ctx, poly)
    sim = _make(bsg, m, 1e-3)
    with pytest.raises(bsg.BsgError, match="interior face connects two segments"):
        sim.set_segments([0, m.n_cells // 2, m.n_cells], [1e-3, 1e-3])
    sim.close()
    m.close()
