"""Locality renumbering of arbitrarily numbered meshes (reverse Cuthill-McKee inside the library,
the caller's numbering kept at the ABI).

The 8^3 jittered-Voronoi fixture mesh with its cells numbered at random: the library renumbers it
internally, and every result comes back in the caller's (shuffled) numbering.  Mapped back to the
fixture's numbering, the converged SIMPLE fields after the reference's own number of outer
iterations agree with the reference's to 1e-8 (the renumbered cells traverse their faces in
another order, so sums round differently; nothing else changes), and the geometry to 1e-12.  The
pressure is anchored at the caller's cell 0, as the reference anchors it, so after the shuffle it
agrees up to the constant that moves the anchor to another cell.
"""
import numpy as np
import pytest

from helpers import Golden, fields_at_reference_count, rel_l2
from test_meshgen import shuffled

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def test_shuffled_mesh_is_renumbered_and_results_come_back_in_caller_order(ctx):
    import babelsim_b200 as bsg
    from babelsim_b200.api import locality_order
    g = Golden("voronoi8_config2")
    sh, perm = shuffled(g.poly)
    assert locality_order(sh)[1]
    m = bsg.Mesh.from_polyhedral(ctx, sh)
    ref = g.ref_geometry()
    xc = m.export("cell_centres").reshape(-1, 3)[perm]
    assert np.max(np.abs(xc - ref["cell_centres"].reshape(-1, 3))) <= 1e-12
    V = m.export("cell_volumes")[perm]
    assert np.max(np.abs(V - ref["cell_volumes"])) <= 1e-12 * np.max(ref["cell_volumes"])
    assert np.array_equal(m.export("face_owner"), sh.owner)
    host = bsg.Mesh.from_polyhedral(ctx, sh, host_geometry=True)
    assert np.array_equal(host.export("cell_centres"), m.export("cell_centres"))
    host.close()
    s = g.settings()
    sol = g.meta["solution"]

    def make():
        sim = bsg.Simple(m, s.rho, s.mu, s.alpha_u, s.alpha_p, s.non_orthogonal_corrections, s.mass_tolerance,
                         s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
                         bsg.options(**s.momentum), bsg.options(**s.pressure),
                         bsg.solver_config("bcgs", "bjacobi", sol["equation.momentum.absoluteTolerance"],
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
    assert rel_l2(U[perm], g["U_conv"]) < 1e-8
    # the pressure level is anchored at the caller's cell 0 (reference(Equation, cell 0, value)),
    # which the shuffle made another cell: equal up to that constant
    j0 = int(np.flatnonzero(perm == 0)[0])
    ref_p = g["p_conv"] - g["p_conv"][j0]
    assert abs(p[0]) <= 1e-6 * np.max(np.abs(p))
    assert rel_l2(p[perm] - p[0], ref_p) < 1e-8
    m.close()


def test_shuffled_linear_system_through_the_seam(ctx):
    """bsg_solve_ldu on a renumbered mesh: diagonal, source and x in the caller's numbering."""
    import babelsim_b200 as bsg
    import scipy.sparse.linalg as spla
    from helpers import ref_system_groups
    from oracle import fvm
    g = Golden("voronoi8_config2")
    sh, perm = shuffled(g.poly)
    m = bsg.Mesh.from_polyhedral(ctx, sh)
    sysp = ref_system_groups(g)[0]["pressure"][0]
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    diag, src = sysp["diag"][inv], sysp["source"][inv]   # shuffled cell c' holds fixture cell inv[c']
    x, res = bsg.solve_ldu(m, bsg.solver_config("cg", "hypre", 1e-30, 1e-12, 2000), diag, sysp["upper"],
                           sysp["lower"], src)
    assert res[0].status == 0
    ldu = fvm.LDU(g.oracle_geometry(), False)
    ldu.diag, ldu.upper, ldu.lower, ldu.source = sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"]
    exact = spla.spsolve(ldu.matrix().tocsc(), ldu.source)
    assert rel_l2(x[perm], exact) < 1e-8
    m.close()
