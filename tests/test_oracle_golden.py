"""The oracle restatement pinned against the reference's own sources (golden fixtures).

The fixtures come from tests/golden/make_golden.py, which runs the reference's
unmodified finite-volume sources and SIMPLE loop (compiled serially by
oracle/ref).  Tolerances: assembled coefficients 1e-12 relative; fields after
one iteration from the reference's own state 1e-9 (the reference's Krylov
solves stop at rtol 1e-12, 1e-10 on the Voronoi cubes); converged fields 1e-8
after the reference's own number of outer iterations (outer tolerance 1e-6).
"""
import numpy as np
import pytest

from helpers import (CASES, PISO_CASES, PISO_POTENTIAL_CASES, PISO_RANS_CASES, RANS_CASES, SA_CASES, VORONOI_CASES, Golden,
                     kepsilon_factory, komega_factory, piso_settings, ref_system_groups, rel, rel_l2, sa_factory)
from oracle import fvm, piso, simple


@pytest.mark.parametrize("name", CASES)
def test_geometry_matches_reference(name):
    g = Golden(name)
    geo = g.oracle_geometry()
    ref = g.ref_geometry()
    pairs = [("face_area_vectors", geo.Sf), ("face_centres", geo.xf), ("face_areas", geo.area),
             ("face_normals", geo.normal), ("face_owner_weights", geo.weight),
             ("face_orthogonal_coefficients", geo.dcoef), ("face_non_orthogonal", geo.kvec),
             ("face_skewness", geo.skew), ("cell_centres", geo.xc), ("cell_volumes", geo.volume)]
    for key, mine in pairs:
        r = ref[key].reshape(mine.shape)
        scale = max(np.max(np.abs(r)), 1e-300)
        assert np.max(np.abs(mine - r)) <= 1e-12 * scale + 1e-15, key
    assert geo.orthogonal == bool(ref["orthogonal_geometry"][0])


def _state(g, k):
    n = g.poly.n_cells
    if k == 0:
        return np.zeros((n, 3)), np.zeros(n), None
    return g[f"U_{k}"], g[f"p_{k}"], g[f"phi_{k}"]


@pytest.mark.parametrize("name", ["cavity12_upwind", "warped5_corrected"] + VORONOI_CASES)
def test_one_iteration_systems_and_fields(name):
    g = Golden(name)
    geo = g.oracle_geometry()
    groups = ref_system_groups(g)
    for k in range(1, g.K + 1):
        U0, p0, phi0 = _state(g, k - 1)
        cap = {}

        def capture(it, d):
            cap.update(d)
        st = simple.run_simple(geo, g.U_bcs(), g.p_bcs(), g.settings(), U0=U0, p0=p0, phi0=phi0, iterations=1,
                               capture=capture)
        ref = groups[k - 1]
        mom = cap["momentum_relaxed"]
        for key in ("diag", "upper", "lower", "source"):
            assert rel(getattr(mom, key), ref["momentum"][key].reshape(getattr(mom, key).shape)) < 1e-12, (k, key)
        # the first pressure source is div(phiH) of this iteration's momentum solution: it agrees
        # to the momentum solve's tolerance (1e-12 when that solve ran to rtol 1e-12)
        mom_rtol = g.meta["solution"]["equation.momentum.relativeTolerance"]
        for j, (mine, theirs) in enumerate(zip(cap["pressure"], ref["pressure"])):
            tol = max(1e-12, 100 * mom_rtol) if j == 0 else 1e-8
            for key in ("diag", "upper", "lower"):
                assert rel(getattr(mine, key), theirs[key]) < 1e-12, (k, j, key)
            assert rel(mine.source, theirs["source"]) < tol, (k, j, "source")
        assert rel_l2(st.U, g[f"U_{k}"]) < 1e-9
        assert rel_l2(st.p, g[f"p_{k}"]) < 1e-9
        assert rel_l2(st.phi, g[f"phi_{k}"]) < 1e-9


@pytest.mark.parametrize("name", ["cavity12_upwind", "warped5_corrected", "voronoi8_config2"])
def test_converged_fields(name):
    g = Golden(name)
    st = simple.run_simple(g.oracle_geometry(), g.U_bcs(), g.p_bcs(), g.settings(), iterations=5000)
    assert st.converged
    assert st.iterations == int(g["conv_info"][1])
    assert rel_l2(st.U, g["U_conv"]) < 1e-8
    assert rel_l2(st.p, g["p_conv"]) < 1e-8


def test_operators_known_answers():
    """Analytic answers of the reference's tests/operators_test.cpp:71-104 on a 3x3x3 box."""
    from babelsim_b200 import meshgen
    from oracle import geometry
    pm = meshgen.hex_box(3, 3, 3, (0, 0, 0), (3, 3, 3))
    geo = geometry.compute_geometry(geometry.PolyMesh(pm.vertices, pm.faces, pm.owner, pm.neighbour, pm.patch,
                                                      pm.patch_names, pm.patch_kinds))
    lin = 2.0 * geo.xc[:, 0] - 3.0 * geo.xc[:, 1] + 0.5 * geo.xc[:, 2] + 1.0
    centre = 1 + 3 * (1 + 3 * 1)
    zg = [(fvm.ZERO_GRADIENT, 0.0)] * 6
    f = fvm.Field(geo, lin, zg)
    for method in ("greenGauss", "leastSquares"):
        gr = fvm.gradient(f, method)
        assert np.allclose(gr[centre], [2.0, -3.0, 0.5], atol=1e-12)
    # Least squares is exact for a linear field whose constraints are consistent with
    # it on every patch, boundary cells included (mirror points, operators.cpp:336-347).
    from babelsim_b200 import meshgen as mg
    wp = mg.warped_box(4)
    wgeo = geometry.compute_geometry(geometry.PolyMesh(wp.vertices, wp.faces, wp.owner, wp.neighbour, wp.patch,
                                                       wp.patch_names, wp.patch_kinds))
    xf = fvm.Field(wgeo, wgeo.xc[:, 0].copy(), [(fvm.FIXED_VALUE, 0.0), (fvm.FIXED_VALUE, 1.0)] +
                   [(fvm.ZERO_GRADIENT, 0.0)] * 4)
    assert np.allclose(fvm.gradient(xf, "leastSquares"), [1.0, 0.0, 0.0], atol=1e-12)
    U = fvm.Field(geo, geo.xc.copy(), [(fvm.ZERO_GRADIENT, np.zeros(3))] * 6)
    phi = fvm.flux(U, "linear", "greenGauss")
    assert abs(fvm.divergence_flux(geo, phi)[centre] - 3.0) < 1e-12
    quad = fvm.Field(geo, np.sum(geo.xc ** 2, axis=1), zg)
    eq = fvm.LDU(geo, False)
    fvm.add_diffusion(eq, np.ones(geo.n_faces), quad, None, "orthogonal")
    lap = -(eq.apply(quad.v) - eq.source) / geo.volume   # -(A x - b) / V = laplacian
    assert abs(lap[centre] - 6.0) < 1e-12


@pytest.mark.parametrize("name", PISO_CASES)
def test_piso_steps_match_reference(name):
    """The PISO restatement reproduces the reference's runPiso after every time step
    (BDF2 with a shortened last step, and Euler with non-orthogonal correctors)."""
    from oracle import piso
    g = Golden(name)
    geo = g.oracle_geometry()
    st = piso.run_piso(geo, g.U_bcs(), g.p_bcs(), piso_settings(g), steps=1)
    assert st.steps == 1
    for k in range(1, g.K + 1):
        st = piso.run_piso(geo, g.U_bcs(), g.p_bcs(), piso_settings(g, g.meta["ends"][k - 1]))
        assert st.status == "completed" and st.steps == k
        assert rel_l2(st.U, g[f"U_{k}"]) <= 1e-10, k
        assert rel_l2(st.p, g[f"p_{k}"]) <= 1e-10, k
        assert rel_l2(st.phi, g[f"phi_{k}"]) <= 1e-10, k


def test_bdf2_weights_variable_step():
    """Variable-step BDF2 weights (procedural_equation.cpp:205-214) reduce to the constant-step
    1.5/2/-0.5 form and integrate a quadratic exactly."""
    from oracle import piso
    dt = 0.1
    a0, a1, a2 = piso.time_weights("bdf2", dt, dt)
    assert np.allclose([a0 * dt, a1 * dt, a2 * dt], [1.5, 2.0, -0.5])
    # exactness on y(t) = t^2 with steps h1 (older) and h0 (current)
    h1, h0 = 0.3, 0.12
    a0, a1, a2 = piso.time_weights("bdf2", h0, h1)
    t0 = 1.0
    y = lambda t: t * t
    assert abs(a0 * y(t0) - a1 * y(t0 - h0) - a2 * y(t0 - h0 - h1) - 2 * t0) < 1e-12


@pytest.mark.parametrize("name", RANS_CASES + ["kepsilon_channel"])
def test_komega_simple_iterations_match_reference(name):
    """SIMPLE with the Wilcox-1988m k-omega model: the restatement (calculated boundary traces of
    mut/muEff/diffusivities, stress remainder divergence, omega-then-k transport with bounding)
    reproduces the reference's U, p, phi, k, omega, mut after every outer iteration."""
    g = Golden(name)
    geo = g.oracle_geometry()
    s = g.settings()
    s.mu = g.meta["physics"]["dynamicViscosity"]
    for k in range(1, g.K + 1):
        model = kepsilon_factory(g) if name.startswith("kepsilon") else komega_factory(g)
        st = simple.run_simple(geo, g.U_bcs(), g.p_bcs(), s, iterations=k, turbulence=model)
        for key, mine in (("U", st.U), ("p", st.p), ("phi", st.phi), ("k", st.k), ("omega", st.omega),
                          ("mut", st.mut)):
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-9, (key, k)


@pytest.mark.parametrize("name", SA_CASES)
def test_spalart_allmaras_simple_iterations_match_reference(name):
    """SIMPLE with the Spalart-Allmaras model (given wall distance): the restatement of the closure
    functions, the implicit/explicit split of the net reaction, the cb2 gradient source and the calculated
    traces of mut/muEff/diffusivity reproduces the reference's U, p, phi, nuTilda, mut every iteration."""
    g = Golden(name)
    geo = g.oracle_geometry()
    s = g.settings()
    s.mu = g.meta["physics"]["dynamicViscosity"]
    for k in range(1, g.K + 1):
        st = simple.run_simple(geo, g.U_bcs(), g.p_bcs(), s, iterations=k, turbulence=sa_factory(g))
        for key, mine in (("U", st.U), ("p", st.p), ("phi", st.phi), ("nuTilda", st.nuTilda), ("mut", st.mut)):
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-9, (key, k, rel_l2(mine, g[f"{key}_{k}"]))


@pytest.mark.parametrize("name", PISO_RANS_CASES)
def test_piso_with_turbulence_matches_reference(name):
    """runPiso with an eddy-viscosity model: transient model histories saved once per step, ddt ahead
    of convection in the transport equations, transport corrected at each time level until
    turbulenceTolerance; U, p, phi and the model fields after every step."""
    g = Golden(name)
    geo = g.oracle_geometry()
    if "_sa_" in name:
        model, keys = sa_factory(g), {"nuTilda": "nuTilda", "mut": "mut"}
    elif "kepsilon" in name:
        model, keys = kepsilon_factory(g), {"k": "k", "epsilon": "omega", "mut": "mut"}
    else:
        model, keys = komega_factory(g), {"k": "k", "omega": "omega", "mut": "mut"}
    for k in range(1, g.K + 1):
        st = piso.run_piso(geo, g.U_bcs(), g.p_bcs(), piso_settings(g, g.meta["ends"][k - 1]), turbulence=model)
        assert st.status == "completed"
        for key, mine in [("U", st.U), ("p", st.p), ("phi", st.phi)] + [(f, getattr(st, a)) for f, a in keys.items()]:
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-9, (key, k, rel_l2(mine, g[f"{key}_{k}"]))


@pytest.mark.parametrize("name", PISO_POTENTIAL_CASES)
def test_piso_potential_flow_start_matches_reference(name):
    """initializePotentialFlow: potential solves on the initial flux imbalance (homogeneous pressure
    constraints, unit diffusivity), U -= grad(pPrime), phi += faceFlux; then the normal time steps."""
    g = Golden(name)
    geo = g.oracle_geometry()
    for k in range(1, g.K + 1):
        st = piso.run_piso(geo, g.U_bcs(), g.p_bcs(), piso_settings(g, g.meta["ends"][k - 1]))
        assert st.status == "completed"
        for key, mine in (("U", st.U), ("p", st.p), ("phi", st.phi)):
            assert rel_l2(mine, g[f"{key}_{k}"]) <= 1e-9, (key, k, rel_l2(mine, g[f"{key}_{k}"]))


def test_vorticity_magnitude_known_answers():
    """sqrt(2 W:W) is the vorticity magnitude: 2w for a solid rotation at angular rate w, zero for pure strain."""
    from oracle import rans
    w = 1.7
    rot = np.array([[[0.0, -w, 0.0], [w, 0.0, 0.0], [0.0, 0.0, 0.0]]])
    strain = np.array([[[1.0, 2.0, 0.0], [2.0, -1.0, 0.0], [0.0, 0.0, 0.0]]])
    assert abs(rans.vorticity_magnitude(rot)[0] - 2.0 * w) < 1e-15
    assert rans.vorticity_magnitude(strain)[0] == 0.0


def test_strain_squared_known_answers():
    """2 dev(symm G):dev(symm G): zero for solid rotation and isotropic expansion; 2 (a^2/2) for shear."""
    from oracle import rans
    rot = np.array([[[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 0.0]]])
    iso = np.eye(3)[None] * 2.5
    a = 3.0
    shear = np.zeros((1, 3, 3))
    shear[0, 0, 1] = a
    assert abs(rans.strain_squared(rot)[0]) < 1e-15
    assert abs(rans.strain_squared(iso)[0]) < 1e-14
    assert abs(rans.strain_squared(shear)[0] - a * a) < 1e-14
