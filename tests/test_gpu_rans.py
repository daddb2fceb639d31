"""k-omega, k-epsilon and Spalart-Allmaras SIMPLE on the GPU vs the reference's own runSimple +
KOmega / KEpsilon / SpalartAllmaras, through the C ABI.

Tolerance: 1e-8 relative L2 on U, p, phi, k, omega (epsilon) and mut after every outer
iteration (every linear solve at rtol 1e-12 on both sides; the transported
turbulence equations are non-symmetric and run BiCGStab with Jacobi here,
against the reference's Krylov backend at the same tolerance).
"""
import numpy as np
import pytest

from helpers import RANS_CASES, SA_CASES, Golden, komega_constants, rel_l2
from oracle import fvm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def _solver(bsg, sol, eq, ksp, pc, max_it=20000):
    return bsg.solver_config(ksp, pc, sol[f"equation.{eq}.absoluteTolerance"], sol[f"equation.{eq}.relativeTolerance"],
                             max_it)


def _komega_simple(bsg, g, m, pc="hypre"):
    s = g.settings()
    ph, sol, meth = g.meta["physics"], g.meta["solution"], g.meta["methods"]
    sim = bsg.Simple(m, ph["density"], ph["dynamicViscosity"], s.alpha_u, s.alpha_p, s.non_orthogonal_corrections,
                     s.mass_tolerance, s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
                     bsg.options(**s.momentum), bsg.options(**s.pressure),
                     _solver(bsg, sol, "momentum", "bcgs", "bjacobi", 2000),
                     _solver(bsg, sol, "pressureCorrection", "cg", pc))
    second = g.meta.get("second", "omega")
    if second == "epsilon":
        sim.enable_kepsilon(ph["kEpsilonCmu"], ph["kEpsilonC1"], ph["kEpsilonC2"], ph["kEpsilonSigmaK"],
                            ph["kEpsilonSigmaEpsilon"], ph["kMin"], ph["epsilonMin"], sol["turbulenceRelaxation"],
                            sol["turbulenceTolerance"], bsg.options(**meth["kTransport"]),
                            bsg.options(**meth["epsilonTransport"]),
                            _solver(bsg, sol, "kTransport", "bcgs", "bjacobi", 2000),
                            _solver(bsg, sol, "epsilonTransport", "bcgs", "bjacobi", 2000))
    else:
        c = komega_constants(g)
        sim.enable_komega(c.beta_star, c.beta, c.gamma, c.sigma_k, c.sigma_omega, c.k_min, c.omega_min,
                          c.viscosity_ratio_max, c.relaxation, c.tolerance, bsg.options(**meth["kTransport"]),
                          bsg.options(**meth["omegaTransport"]),
                          _solver(bsg, sol, "kTransport", "bcgs", "bjacobi", 2000),
                          _solver(bsg, sol, "omegaTransport", "bcgs", "bjacobi", 2000))
    for p, (t, v) in enumerate(g.meta["U_bcs"]):
        sim.set_boundary("U", p, t, v)
    for p, (t, v) in enumerate(g.meta["p_bcs"]):
        sim.set_boundary("p", p, t, v)
    for p, (t, v) in enumerate(g.meta["k_bcs"]):
        sim.set_boundary("k", p, t, v)
    for p, (t, v) in enumerate(g.meta["omega_bcs"]):
        sim.set_boundary(second, p, t, v)
    n = m.n_cells
    sim.set_turbulence_fields(np.full(n, g.meta["k_internal"]), np.full(n, g.meta["omega_internal"]))
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    return sim


@pytest.mark.parametrize("name", RANS_CASES + ["kepsilon_channel"])
def test_komega_simple_every_iteration_matches_reference(ctx, name):
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sim = _komega_simple(bsg, g, m)
    for k in range(1, g.K + 1):
        r = sim.iterate(1)
        assert r.status != 2 and r.iterations == k
        U, p, phi = sim.fields()
        kk, w, mut = sim.turbulence_fields()
        for key, mine in (("U", U), ("p", p), ("phi", phi), ("k", kk), ("omega", w), ("mut", mut)):
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-8, (key, k)
        assert np.isfinite(r.turbulence_change) and r.turbulence_residual > 0
    sim.close()
    m.close()


@pytest.mark.parametrize("name", SA_CASES)
def test_spalart_allmaras_simple_every_iteration_matches_reference(ctx, name):
    """One-equation model with a given wall distance: U, p, phi, nuTilda and mut after every outer
    iteration within 1e-8 of the reference (linear solves at rtol 1e-12 on both sides)."""
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    s = g.settings()
    ph, sol, meth = g.meta["physics"], g.meta["solution"], g.meta["methods"]
    sim = bsg.Simple(m, ph["density"], ph["dynamicViscosity"], s.alpha_u, s.alpha_p, s.non_orthogonal_corrections,
                     s.mass_tolerance, s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
                     bsg.options(**s.momentum), bsg.options(**s.pressure),
                     _solver(bsg, sol, "momentum", "bcgs", "bjacobi", 2000),
                     _solver(bsg, sol, "pressureCorrection", "cg", "hypre"))
    sim.enable_spalart_allmaras(ph["saCb1"], ph["saCb2"], ph["saSigma"], ph["saKappa"], 0.0, ph["saCw2"],
                                ph["saCw3"], ph["saCv1"], ph["saCt3"], ph["saCt4"], ph["saNuTildaMin"],
                                ph["saWallDistanceMin"], sol["turbulenceRelaxation"], sol["turbulenceTolerance"],
                                bsg.options(**meth["nuTildaTransport"]),
                                _solver(bsg, sol, "nuTildaTransport", "bcgs", "bjacobi", 2000))
    for p, (t, v) in enumerate(g.meta["U_bcs"]):
        sim.set_boundary("U", p, t, v)
    for p, (t, v) in enumerate(g.meta["p_bcs"]):
        sim.set_boundary("p", p, t, v)
    for p, (t, v) in enumerate(g.meta["nuTilda_bcs"]):
        sim.set_boundary("nuTilda", p, t, v)
    n = m.n_cells
    sim.set_wall_distance(g["wall_distance"])
    sim.set_turbulence_fields(None, np.full(n, g.meta["nuTilda_internal"]))
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    for k in range(1, g.K + 1):
        r = sim.iterate(1)
        assert r.status != 2 and r.iterations == k
        U, p, phi = sim.fields()
        kk, nt, mut = sim.turbulence_fields()
        assert kk is None
        for key, mine in (("U", U), ("p", p), ("phi", phi), ("nuTilda", nt), ("mut", mut)):
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-8, (key, k, rel_l2(mine, g[f"{key}_{k}"]))
        assert np.isfinite(r.turbulence_change) and r.turbulence_residual > 0
    sim.close()
    m.close()


def test_scalar_bicgstab_on_a_nonsymmetric_system(ctx):
    """kspType bcgs on a scalar convection-diffusion system (the transported-turbulence shape)
    through the linear-system seam, against a direct solve."""
    import babelsim_b200 as bsg
    import scipy.sparse.linalg as spla
    g = Golden("komega_warped5")
    geo = g.oracle_geometry()
    rng = np.random.default_rng(5)
    x = fvm.Field(geo, rng.random(geo.n_cells), [(fvm.FIXED_VALUE, 1.0)] * 6, flux=None)
    phi = 0.5 * rng.standard_normal(geo.n_faces)
    eq = fvm.Equation(x, dict(interpolation="linear", gradient="greenGauss", convection="upwind",
                              diffusion="orthogonal"), {})
    fvm.eq_div(eq, phi, 1.0)
    fvm.eq_laplacian(eq, 0.05, -1.0)
    q = eq.ldu
    q.diag = q.diag + 2.0 * geo.volume
    q.source = q.source + geo.volume * rng.random(geo.n_cells)
    exact = spla.spsolve(q.matrix().tocsc(), q.source)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sol, res = bsg.solve_ldu(m, bsg.solver_config("bcgs", "bjacobi", 1e-30, 1e-12, 2000), q.diag, q.upper, q.lower,
                             q.source)
    assert res[0].status == 0
    assert rel_l2(sol, exact) < 1e-9
    m.close()
