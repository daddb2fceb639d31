"""CUDA path vs the oracle and the reference's golden fixtures, through the C ABI.

Tolerances (relative): geometry 1e-12; explicit operators and assembled LDU
coefficients 1e-12 (FP64, different summation order only); linear solves at
rtol 1e-12 vs a direct solve 1e-8; one SIMPLE iteration from the reference's
own state 1e-9; converged SIMPLE fields 1e-8 after the reference's own number of
outer iterations (outer tolerance 1e-6; solver tolerance 1e-10 on the Voronoi
cubes, 1e-12 elsewhere).  The jittered-Voronoi cubes (10-16 faces per cell,
least-squares gradients, corrected diffusion, linearUpwind, 2 non-orthogonal
correctors) are the 1M-cell bench workload's mesh class and settings.
"""
import numpy as np
import pytest

from helpers import CASES, VORONOI_CASES, Golden, fields_at_reference_count, ref_system_groups, rel, rel_l2
from oracle import fvm, simple

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import babelsim_b200 as bsg
    c = bsg.Context(0)
    yield c
    c.close()


def device_mesh(ctx, g):
    import babelsim_b200 as bsg
    return bsg.Mesh.from_polyhedral(ctx, g.poly)


@pytest.mark.parametrize("name", CASES)
def test_geometry(ctx, name):
    g = Golden(name)
    m = device_mesh(ctx, g)
    ref = g.ref_geometry()
    for key in ("face_area_vectors", "face_centres", "face_areas", "face_normals", "face_owner_weights",
                "face_orthogonal_coefficients", "face_non_orthogonal", "face_skewness", "cell_centres",
                "cell_volumes"):
        mine = m.export(key)
        r = ref[key].reshape(mine.shape)
        assert np.max(np.abs(mine - r)) <= 1e-12 * max(np.max(np.abs(r)), 1e-300) + 1e-15, key
    assert m.orthogonal == bool(ref["orthogonal_geometry"][0])


def _mixed_bcs(kind):
    # one of each constraint over the six patches of a box
    if kind == "scalar":
        return [("fixedValue", 1.5), ("fixedGradient", -0.7), ("zeroGradient", 0.0), ("inletOutlet", 2.0),
                ("symmetry", 0.0), ("fixedValue", -0.25)]
    return [("fixedValue", (1.0, 0.5, 0.0)), ("fixedGradient", (0.1, -0.2, 0.3)), ("zeroGradient", (0, 0, 0)),
            ("inletOutlet", (0.0, -1.0, 0.2)), ("symmetry", (0, 0, 0)), ("fixedValue", (0.0, 0.0, 1.0))]


def _fields(ctx, g, seed=3):
    """A device mesh plus matching oracle/device scalar and vector fields with mixed constraints."""
    import babelsim_b200 as bsg
    rng = np.random.default_rng(seed)
    geo = g.oracle_geometry()
    m = device_mesh(ctx, g)
    n = geo.n_cells
    xs = np.sin(3 * geo.xc[:, 0]) + geo.xc[:, 1] ** 2 + 0.1 * rng.standard_normal(n)
    xv = np.stack([np.cos(2 * geo.xc[:, 1]), geo.xc[:, 0] * geo.xc[:, 2], geo.xc[:, 2]], 1) + \
        0.05 * rng.standard_normal((n, 3))
    flux = rng.standard_normal(geo.n_faces)
    sb, vb = _mixed_bcs("scalar"), _mixed_bcs("vector")
    os_ = fvm.Field(geo, xs, [(fvm.BC_NAMES[t], v) for t, v in sb], flux=flux)
    ov = fvm.Field(geo, xv, [(fvm.BC_NAMES[t], np.array(v, float)) for t, v in vb], flux=flux)
    phi = bsg.Field(m, "face", 1, flux)
    ds = bsg.Field(m, "cell", 1, xs)
    dv = bsg.Field(m, "cell", 3, xv)
    for p, (t, v) in enumerate(sb):
        ds.set_boundary(p, t, v)
    for p, (t, v) in enumerate(vb):
        dv.set_boundary(p, t, v)
    ds.set_boundary_flux(phi)
    dv.set_boundary_flux(phi)
    return geo, m, os_, ov, ds, dv, phi, flux


@pytest.mark.parametrize("name", ["warped5_corrected", "cavity12_upwind"])
def test_explicit_operators(ctx, name):
    import babelsim_b200 as bsg
    g = Golden(name)
    geo, m, os_, ov, ds, dv, phi, flux = _fields(ctx, g)
    for method in ("greenGauss", "leastSquares"):
        assert rel(bsg.grad(ds, method).download(), fvm.gradient(os_, method)) < 1e-12, method
        mine = bsg.grad(dv, method).download().reshape(-1, 3, 3)
        assert rel(mine, fvm.gradient(ov, method)) < 1e-12, method
    for interp in ("linear", "corrected"):
        o = bsg.options(interpolation=interp, gradient="leastSquares")
        assert rel(bsg.interpolate(ds, o).download(), fvm.interpolate(os_, interp, "leastSquares")) < 1e-12
        assert rel(bsg.interpolate(dv, o).download(), fvm.interpolate(ov, interp, "leastSquares")) < 1e-12
    assert rel(bsg.div_flux(phi).download(), fvm.divergence_flux(geo, flux)) < 1e-12
    for diff in ("orthogonal", "corrected", "limitedCorrected"):
        o = bsg.options(gradient="greenGauss", diffusion=diff)
        gref = fvm.gradient(os_, "greenGauss")
        assert rel(bsg.normal_gradient(ds, o).download(), fvm.normal_gradient(os_, gref, diff)) < 1e-12, diff


@pytest.mark.parametrize("conv", ["upwind", "linearUpwind", "central"])
@pytest.mark.parametrize("diff", ["orthogonal", "corrected", "limitedCorrected"])
def test_assembly(ctx, conv, diff):
    """equ::div + equ::laplacian + source + relax + scale on mixed constraints, scalar and vector."""
    import babelsim_b200 as bsg
    g = Golden("warped5_corrected")
    geo, m, os_, ov, ds, dv, phi, flux = _fields(ctx, g, seed=11)
    interp = "corrected" if conv == "central" else "linear"
    for of, df in ((os_, ds), (ov, dv)):
        opts = dict(interpolation=interp, gradient="leastSquares", convection=conv, diffusion=diff)
        eq = fvm.Equation(of.copy(), opts, {})
        gamma = 0.3 + np.abs(np.sin(geo.xc[:, 0]))
        kfield = fvm.Field(geo, gamma, [(fvm.ZERO_GRADIENT, 0.0)] * 6)
        fvm.eq_div(eq, flux, 1.3)
        fvm.eq_laplacian(eq, kfield, -1.0)
        src = np.cos(geo.xc[:, 1]) if not of.vector else np.stack([geo.xc[:, 1], -geo.xc[:, 0], geo.xc[:, 2]], 1)
        fvm.eq_source(eq, src, -0.5)
        prev = of.v * 0.9
        fvm.eq_relax(eq, prev, 0.7)
        fvm.eq_scale(eq, 0.7)
        o = bsg.options(**opts)
        deq = bsg.Equation(df, o)
        deq.div(phi, 1.3)
        kdev = bsg.Field(m, "cell", 1, gamma)
        deq.laplacian(kdev, -1.0)
        deq.source(bsg.Field(m, "cell", of.v.shape[1] if of.vector else 1, src), -0.5)
        deq.relax(bsg.Field(m, "cell", 3 if of.vector else 1, prev), 0.7)
        deq.scale(0.7)
        got = deq.download()
        for key in ("diag", "upper", "lower", "source"):
            assert rel(got[key], getattr(eq.ldu, key)) < 1e-12, (of.vector, key)
        if not of.vector:
            sol = np.sin(geo.xc[:, 2])
            assert rel(deq.face_flux(bsg.Field(m, "cell", 1, sol)).download(), fvm.eq_face_flux(eq, sol)) < 1e-12


@pytest.mark.parametrize("name", ["cavity12_upwind", "warped5_corrected"] + VORONOI_CASES)
def test_simple_iteration_systems(ctx, name):
    """Momentum and pressure systems of iteration k assembled on the GPU from the reference's state k-1."""
    import babelsim_b200 as bsg
    g = Golden(name)
    geo = g.oracle_geometry()
    m = device_mesh(ctx, g)
    s = g.settings()
    groups = ref_system_groups(g)
    mo = bsg.options(**s.momentum)
    po = bsg.options(**s.pressure)
    for k in range(1, g.K + 1):
        n = geo.n_cells
        U0 = np.zeros((n, 3)) if k == 1 else g[f"U_{k - 1}"]
        p0 = np.zeros(n) if k == 1 else g[f"p_{k - 1}"]
        cap = {}
        simple.run_simple(geo, g.U_bcs(), g.p_bcs(), s, U0=U0, p0=p0,
                          phi0=None if k == 1 else g[f"phi_{k - 1}"], iterations=1, capture=lambda it, d: cap.update(d))
        phi = bsg.Field(m, "face", 1, np.zeros(geo.n_faces) if k == 1 else g[f"phi_{k - 1}"])
        U = bsg.Field(m, "cell", 3, U0)
        for p, (t, v) in enumerate(g.meta["U_bcs"]):
            U.set_boundary(p, t, v)
        mom = bsg.Equation(U, mo)
        mom.div(phi, s.rho)
        mom.laplacian(bsg.Field(m, "cell", 1, np.full(n, s.mu)), -1.0)
        pf = bsg.Field(m, "cell", 1, p0)
        for p, (t, v) in enumerate(g.meta["p_bcs"]):
            pf.set_boundary(p, t, v)
        gp = bsg.grad(pf, s.pressure["gradient"])
        mom.source(bsg.Field(m, "cell", 3, gp.download()), -1.0)
        mom.relax(bsg.Field(m, "cell", 3, U0), s.alpha_u)
        mom.scale(s.alpha_u)
        got = mom.download()
        ref = groups[k - 1]["momentum"]
        for key in ("diag", "upper", "lower", "source"):
            assert rel(got[key], ref[key].reshape(got[key].shape)) < 1e-12, (k, key)
        # first pressure-correction system from the oracle's rAU and div(phiH)
        pp = bsg.Field(m, "cell", 1)
        for p, (t, v) in enumerate(fvm.homogeneous_bcs(g.p_bcs())):
            pp.set_boundary(p, {0: "fixedValue", 2: "zeroGradient", 4: "symmetry"}[t], 0.0)
        peq = bsg.Equation(pp, po)
        peq.laplacian(bsg.Field(m, "cell", 1, cap["rAU"]), -1.0)
        peq.source(bsg.Field(m, "cell", 1, fvm.divergence_flux(geo, cap["phiH"])), -1.0)
        peq.reference_if_unanchored(0.0)
        got = peq.download()
        ref = groups[k - 1]["pressure"][0]
        for key in ("diag", "upper", "lower"):
            assert rel(got[key], ref[key]) < 1e-12, (k, key)
        # div(phiH) of this iteration's momentum solution: as close as that solve's tolerance
        mom_rtol = g.meta["solution"]["equation.momentum.relativeTolerance"]
        assert rel(got["source"], ref["source"]) < max(1e-10, 100 * mom_rtol), k


@pytest.mark.parametrize("pc", ["jacobi", "hypre"])
def test_pressure_solve(ctx, pc):
    """CG with Jacobi or the device AMG on the reference's pressure system, vs a direct solve."""
    import babelsim_b200 as bsg
    import scipy.sparse.linalg as spla
    g = Golden("cavity64_config1")
    m = device_mesh(ctx, g)
    sysp = ref_system_groups(g)[0]["pressure"][0]
    geo = g.oracle_geometry()
    ldu = fvm.LDU(geo, False)
    ldu.diag, ldu.upper, ldu.lower, ldu.source = sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"]
    exact = spla.spsolve(ldu.matrix().tocsc(), ldu.source)
    cfg = bsg.solver_config("cg", pc, 1e-30, 1e-12, 20000)
    x, res = bsg.solve_ldu(m, cfg, sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"])
    assert res[0].status == 0
    assert rel_l2(x, exact) < 1e-8
    assert res[0].final_residual <= 1e-12 * np.linalg.norm(sysp["source"]) * 1.0000001


def test_momentum_solve(ctx):
    import babelsim_b200 as bsg
    import scipy.sparse.linalg as spla
    g = Golden("cavity64_config1")
    m = device_mesh(ctx, g)
    s = ref_system_groups(g)[0]["momentum"]
    geo = g.oracle_geometry()
    ldu = fvm.LDU(geo, True)
    ldu.diag, ldu.upper, ldu.lower = s["diag"], s["upper"], s["lower"]
    b = s["source"].reshape(-1, 3)
    lu = spla.splu(ldu.matrix().tocsc())
    exact = np.stack([lu.solve(b[:, c].copy()) for c in range(3)], 1)
    cfg = bsg.solver_config("bcgs", "bjacobi", 1e-30, 1e-12, 2000)
    x, res = bsg.solve_ldu(m, cfg, s["diag"], s["upper"], s["lower"], b)
    for c in range(3):
        assert res[c].status == 0
    assert rel_l2(x, exact) < 1e-9


def _simple(ctx, g, m, pc="jacobi"):
    import babelsim_b200 as bsg
    s = g.settings()
    sol = g.meta["solution"]
    sim = bsg.Simple(m, s.rho, s.mu, s.alpha_u, s.alpha_p, s.non_orthogonal_corrections, s.mass_tolerance,
                     s.velocity_tolerance, s.momentum_tolerance, s.pressure_tolerance,
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


@pytest.mark.parametrize("name", ["cavity12_upwind", "warped5_corrected"] + VORONOI_CASES)
def test_simple_one_iteration_from_reference_state(ctx, name):
    g = Golden(name)
    m = device_mesh(ctx, g)
    for k in range(1, g.K + 1):
        sim = _simple(ctx, g, m)
        n = m.n_cells
        sim.set_fields(np.zeros((n, 3)) if k == 1 else g[f"U_{k - 1}"], np.zeros(n) if k == 1 else g[f"p_{k - 1}"])
        if k > 1:
            sim.set_flux(g[f"phi_{k - 1}"])
        sim.iterate(1)
        U, p, phi = sim.fields()
        assert rel_l2(U, g[f"U_{k}"]) < 1e-9, k
        assert rel_l2(p, g[f"p_{k}"]) < 1e-9, k
        assert rel_l2(phi, g[f"phi_{k}"]) < 1e-9, k
        sim.close()


@pytest.mark.parametrize("name,pc", [("cavity12_upwind", "jacobi"), ("warped5_corrected", "hypre"),
                                     ("cavity64_config1", "hypre"), ("voronoi8_config2", "hypre"),
                                     ("voronoi8_config2", "jacobi")])
def test_simple_converged(ctx, name, pc):
    g = Golden(name)
    m = device_mesh(ctx, g)
    target = int(g["conv_info"][1])
    r, U, p = fields_at_reference_count(lambda: _simple(ctx, g, m, pc), m.n_cells, target)
    assert r.converged
    assert abs(r.iterations - target) <= 2
    assert rel_l2(U, g["U_conv"]) < 1e-8
    assert rel_l2(p, g["p_conv"]) < 1e-8
