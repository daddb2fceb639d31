"""Transient path on the GPU vs the reference's own runPiso and the oracle, through the C ABI.

Tolerances (relative L2): transient assembly terms 1e-12 (FP64, summation order
only); fields after every PISO time step 1e-8 (linear solves at rtol 1e-12
against the reference's Krylov solves at the same tolerance).
"""
import numpy as np
import pytest

from helpers import PISO_CASES, PISO_POTENTIAL_CASES, PISO_RANS_CASES, Golden, komega_constants, piso_settings, rel_l2
from oracle import fvm, piso

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def _piso(ctx, g, m, pc="hypre"):
    import babelsim_b200 as bsg
    s = piso_settings(g)
    sol = g.meta["solution"]
    sim = bsg.Piso(m, s.rho, s.mu, s.alpha_u, s.max_iterations, s.correctors, None, None,
                   s.non_orthogonal_corrections, s.mass_tolerance, s.velocity_tolerance, s.momentum_tolerance,
                   s.pressure_tolerance, s.time, s.start_time, s.end_time, s.delta_t,
                   bsg.options(**s.momentum), bsg.options(**s.pressure),
                   bsg.solver_config("bcgs", "bjacobi", sol["equation.momentum.absoluteTolerance"],
                                     sol["equation.momentum.relativeTolerance"], 2000),
                   bsg.solver_config("cg", pc, sol["equation.pressureCorrection.absoluteTolerance"],
                                     sol["equation.pressureCorrection.relativeTolerance"], 20000))
    for p, (t, v) in enumerate(g.meta["U_bcs"]):
        sim.set_boundary("U", p, t, v)
    for p, (t, v) in enumerate(g.meta["p_bcs"]):
        sim.set_boundary("p", p, t, v)
    return sim


@pytest.mark.parametrize("pc", ["hypre", "jacobi"])
@pytest.mark.parametrize("name", PISO_CASES)
def test_piso_every_step_matches_reference(ctx, name, pc):
    """One time step at a time to the end time: U, p, phi against the reference's runPiso
    (BDF2 with a shortened last step; Euler with corrected diffusion and three correctors)."""
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sim = _piso(ctx, g, m, pc)
    n = m.n_cells
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    for k in range(1, g.K + 1):
        r = sim.advance(1)
        assert r.steps == k and r.accepted
        assert abs(r.time - g.meta["ends"][k - 1]) <= 1e-15
        U, p, phi = sim.fields()
        assert rel_l2(U, g[f"U_{k}"]) <= 1e-8, k
        assert rel_l2(p, g[f"p_{k}"]) <= 1e-8, k
        assert rel_l2(phi, g[f"phi_{k}"]) <= 1e-8, k
        assert r.mass <= 1e-10 and r.correctors == g.meta["solution"]["nCorrectors"]
    assert r.status == 0  # end time reached
    assert sim.advance(5).steps == g.K  # nothing left to do
    sim.close()
    m.close()


def test_piso_run_to_end_in_one_call(ctx):
    import babelsim_b200 as bsg
    g = Golden("piso_cavity12_bdf2")
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sim = _piso(ctx, g, m)
    n = m.n_cells
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    r = sim.advance(1000)
    assert r.status == 0 and r.steps == g.K
    U, p, _ = sim.fields()
    assert rel_l2(U, g[f"U_{g.K}"]) <= 1e-8
    assert rel_l2(p, g[f"p_{g.K}"]) <= 1e-8
    assert 0.0 < r.courant_mean <= r.courant_max
    sim.close()
    m.close()


@pytest.mark.parametrize("method", ["euler", "bdf2"])
@pytest.mark.parametrize("vector", [False, True])
def test_ddt_reaction_apply_residual(ctx, method, vector):
    """equ::ddt (variable-step BDF2), equ::reaction, equ::apply and equ::residual on the
    warped box against the oracle's restatement of procedural_equation.cpp."""
    import babelsim_b200 as bsg
    g = Golden("warped5_corrected")
    geo = g.oracle_geometry()
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    rng = np.random.default_rng(11)
    n = geo.n_cells
    shape = (n, 3) if vector else (n,)
    comps = 3 if vector else 1
    x = rng.standard_normal(shape)
    prev, older = rng.standard_normal(shape), rng.standard_normal(shape)
    cap = 0.5 + rng.random(n)
    react = rng.standard_normal(n)
    phi = rng.standard_normal(geo.n_faces)
    dt, older_dt = 0.05, 0.08
    # oracle
    bcs = [(fvm.FIXED_VALUE, np.zeros(3) if vector else 0.0)] * 6
    ox = fvm.Field(geo, x, bcs, flux=phi)
    oeq = fvm.Equation(ox, dict(interpolation="linear", gradient="leastSquares", convection="upwind",
                                diffusion="corrected"), {})
    fvm.eq_div(oeq, phi, 1.3)
    fvm.eq_laplacian(oeq, 0.7, -1.0)
    hist = piso.History(fvm.Field(geo, older, bcs))
    hist.save(fvm.Field(geo, older, bcs), older_dt)
    hist.save(fvm.Field(geo, prev, bcs), dt)
    a0, a1, a2 = piso.time_weights(method, dt, older_dt)
    w = cap * geo.volume
    q = oeq.ldu
    q.diag = q.diag + w * a0
    q.source = q.source + ((w * a1)[:, None] * prev if vector else (w * a1) * prev)
    if method == "bdf2":
        q.source = q.source + ((w * a2)[:, None] * older if vector else (w * a2) * older)
    q.diag = q.diag + 0.4 * react * geo.volume
    q.diag = q.diag + 2.5 * geo.volume
    # device
    d_x = bsg.Field(m, "cell", comps, x)
    for p in range(6):
        d_x.set_boundary(p, "fixedValue", 0.0)
    d_phi = bsg.Field(m, "face", 1, phi)
    d_x.set_boundary_flux(d_phi)
    eq = bsg.Equation(d_x, bsg.options("linear", "leastSquares", "upwind", "corrected"))
    eq.div(d_phi, 1.3)
    eq.laplacian(0.7, -1.0)
    eq.ddt(bsg.Field(m, "cell", 1, cap), bsg.Field(m, "cell", comps, prev), dt, method,
           bsg.Field(m, "cell", comps, older), older_dt)
    eq.reaction(bsg.Field(m, "cell", 1, react), 0.4)
    eq.reaction(2.5)
    got = eq.download()
    assert np.max(np.abs(got["diag"] - q.diag)) <= 1e-12 * np.max(np.abs(q.diag))
    assert np.max(np.abs(got["source"] - q.source)) <= 1e-12 * np.max(np.abs(q.source))
    y = rng.standard_normal(shape)
    d_y = bsg.Field(m, "cell", comps, y)
    ax = eq.apply(d_y).download()
    ref_ax = q.apply(y)
    assert np.max(np.abs(ax - ref_ax)) <= 1e-12 * np.max(np.abs(ref_ax))
    res = eq.residual(d_y).download()
    assert np.max(np.abs(res - (q.source - ref_ax))) <= 1e-12 * np.max(np.abs(q.source - ref_ax))
    # argument errors are reported, not thrown across the ABI
    with pytest.raises(bsg.BsgError):
        eq.ddt(2.0, bsg.Field(m, "cell", comps, prev), -1.0, method)
    with pytest.raises(bsg.BsgError):
        eq.ddt(bsg.Field(m, "cell", 1, -cap), bsg.Field(m, "cell", comps, prev), dt, "euler")
    if method == "bdf2":
        with pytest.raises(bsg.BsgError):
            eq.ddt(2.0, bsg.Field(m, "cell", comps, prev), dt, "bdf2")  # no older level


@pytest.mark.parametrize("name", PISO_RANS_CASES)
def test_piso_with_turbulence_every_step_matches_reference(ctx, name):
    """runPiso with k-omega or k-epsilon (BDF2) or Spalart-Allmaras (Euler): the model's histories saved each step,
    its transport (with the time term) corrected after the pressure correctors until
    turbulenceTolerance; U, p, phi and the model's fields after every step within 1e-8."""
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sim = _piso(ctx, g, m)
    ph, sol, meth = g.meta["physics"], g.meta["solution"], g.meta["methods"]
    sim.set_turbulence_controls("iterated", sol["turbulenceMaxIterations"], 0)

    def solver(eq):
        return bsg.solver_config("bcgs", "bjacobi", sol[f"equation.{eq}.absoluteTolerance"],
                                 sol[f"equation.{eq}.relativeTolerance"], 2000)
    n = m.n_cells
    sa = "_sa_" in name
    if sa:
        sim.enable_spalart_allmaras(ph["saCb1"], ph["saCb2"], ph["saSigma"], ph["saKappa"], 0.0, ph["saCw2"],
                                    ph["saCw3"], ph["saCv1"], ph["saCt3"], ph["saCt4"], ph["saNuTildaMin"],
                                    ph["saWallDistanceMin"], sol["turbulenceRelaxation"], sol["turbulenceTolerance"],
                                    bsg.options(**meth["nuTildaTransport"]), solver("nuTildaTransport"))
        for p, (t, v) in enumerate(g.meta["nuTilda_bcs"]):
            sim.set_boundary("nuTilda", p, t, v)
        sim.set_wall_distance(g["wall_distance"])
        sim.set_turbulence_fields(None, np.full(n, g.meta["nuTilda_internal"]))
        keys = ("nuTilda", "mut")
    else:
        second = g.meta.get("second", "omega")
        if second == "epsilon":
            sim.enable_kepsilon(ph["kEpsilonCmu"], ph["kEpsilonC1"], ph["kEpsilonC2"], ph["kEpsilonSigmaK"],
                                ph["kEpsilonSigmaEpsilon"], ph["kMin"], ph["epsilonMin"], sol["turbulenceRelaxation"],
                                sol["turbulenceTolerance"], bsg.options(**meth["kTransport"]),
                                bsg.options(**meth["epsilonTransport"]), solver("kTransport"),
                                solver("epsilonTransport"))
        else:
            c = komega_constants(g)
            sim.enable_komega(c.beta_star, c.beta, c.gamma, c.sigma_k, c.sigma_omega, c.k_min, c.omega_min,
                              c.viscosity_ratio_max, c.relaxation, c.tolerance, bsg.options(**meth["kTransport"]),
                              bsg.options(**meth["omegaTransport"]), solver("kTransport"), solver("omegaTransport"))
        for p, (t, v) in enumerate(g.meta["k_bcs"]):
            sim.set_boundary("k", p, t, v)
        for p, (t, v) in enumerate(g.meta["omega_bcs"]):
            sim.set_boundary(second, p, t, v)
        sim.set_turbulence_fields(np.full(n, g.meta["k_internal"]), np.full(n, g.meta["omega_internal"]))
        keys = ("k", second, "mut")
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    for k in range(1, g.K + 1):
        r = sim.advance(1)
        assert r.steps == k and r.accepted and r.turbulence_corrections >= 1
        U, p, phi = sim.fields()
        kk, second, mut = sim.turbulence_fields()
        mine = dict(U=U, p=p, phi=phi, mut=mut, **({"nuTilda": second} if sa else {"k": kk, keys[1]: second}))
        for key in ("U", "p", "phi") + keys:
            assert rel_l2(mine[key], g[f"{key}_{k}"]) <= 1e-8, (key, k, rel_l2(mine[key], g[f"{key}_{k}"]))
        assert r.turbulence_change <= sol["turbulenceTolerance"] and r.turbulence_residual <= sol["turbulenceTolerance"]
    assert r.status == 0
    sim.close()
    m.close()


@pytest.mark.parametrize("pc", ["hypre", "jacobi"])
@pytest.mark.parametrize("name", PISO_POTENTIAL_CASES)
def test_piso_potential_flow_start_matches_reference(ctx, name, pc):
    """initializePotentialFlow: the potential solves before the first step, then every step within 1e-8."""
    import babelsim_b200 as bsg
    g = Golden(name)
    m = bsg.Mesh.from_polyhedral(ctx, g.poly)
    sim = _piso(ctx, g, m, pc)
    sim.initialize_potential_flow(g.meta["solution"].get("initialNonOrthogonalCorrections", -1))
    n = m.n_cells
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    for k in range(1, g.K + 1):
        r = sim.advance(1)
        assert r.steps == k and r.accepted
        U, p, phi = sim.fields()
        for key, mine in (("U", U), ("p", p), ("phi", phi)):
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-8, (key, k, rel_l2(mine, g[f"{key}_{k}"]))
    sim.close()
    m.close()
