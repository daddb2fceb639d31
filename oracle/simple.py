"""Steady SIMPLE outer loop, restated from src/physics/simple/main.cpp:11-131.  TEST INFRASTRUCTURE ONLY.

Laminar (no turbulence model), constant density and viscosity.  Linear systems
are solved directly (sparse LU), which stands in for the reference's Krylov
solves converged to their tolerance: only the converged solution is pinned.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse.linalg as spla

from . import fvm


@dataclass
class SimpleSettings:
    """The SIMPLE controls read at simple/main.cpp:23-31 plus the per-equation options."""
    rho: float = 1.0
    mu: float = 0.01
    alpha_u: float = 0.7
    alpha_p: float = 0.3
    max_iterations: int = 1000
    non_orthogonal_corrections: int = 1
    mass_tolerance: float = 1e-8
    velocity_tolerance: float = 1e-7
    momentum_tolerance: float = 1e-6
    pressure_tolerance: float = 1e-6
    momentum: dict = field(default_factory=lambda: dict(
        interpolation="linear", gradient="greenGauss", convection="upwind", diffusion="orthogonal"))
    pressure: dict = field(default_factory=lambda: dict(
        interpolation="linear", gradient="greenGauss", convection="upwind", diffusion="orthogonal"))


@dataclass
class SimpleState:
    U: np.ndarray
    p: np.ndarray
    phi: np.ndarray
    iterations: int = 0
    converged: bool = False
    history: list = field(default_factory=list)


def _solve(A, b):
    lu = spla.splu(A.tocsc())
    if b.ndim == 2:
        return np.stack([lu.solve(b[:, c].copy()) for c in range(b.shape[1])], axis=1)
    return lu.solve(b.copy())


def run_simple(geo, U_bcs, p_bcs, settings: SimpleSettings, U0=None, p0=None, iterations=None,
               capture=None, phi0=None, turbulence=None) -> SimpleState:
    """runSimple (simple/main.cpp:11-131).  ``capture(iter, dict)`` receives the
    assembled systems of each iteration (momentum after assembly and after
    relax/scale; pressure systems as solved) for parity checks.  ``phi0``
    resumes from a saved face flux instead of flux(U0).  ``turbulence(geo, phi)``
    builds an eddy-viscosity model (oracle.rans.KOmega) before the initial flux,
    as rans::load does (simple/main.cpp:33); its effective viscosity, stress
    remainder and transport solve enter where simple/main.cpp:53-56, 102-110 put them."""
    nc = geo.n_cells
    U = fvm.Field(geo, np.zeros((nc, 3)) if U0 is None else U0, U_bcs)
    p = fvm.Field(geo, np.zeros(nc) if p0 is None else p0, p_bcs)
    mom_opts = dict(settings.momentum)
    p_opts = dict(settings.pressure)
    pressure_solves = 1 if p_opts["diffusion"] == "orthogonal" else settings.non_orthogonal_corrections + 1
    model = turbulence(geo, np.zeros(geo.n_faces)) if turbulence is not None else None
    phi = fvm.flux(U, mom_opts["interpolation"], mom_opts["gradient"])
    if phi0 is not None:
        phi = np.array(phi0, dtype=np.float64)
    mu_field = fvm.Field(geo, np.full(nc, settings.mu), [(fvm.ZERO_GRADIENT, 0.0)] * len(geo.patch_names or U_bcs))
    V = geo.volume
    state = SimpleState(U.v, p.v, phi)
    n_iter = settings.max_iterations if iterations is None else iterations
    for it in range(n_iter):
        U_prev = U.v.copy()
        mom = fvm.Equation(U, mom_opts, {})
        fvm.eq_div(mom, phi, settings.rho)
        fvm.eq_laplacian(mom, model.effective_viscosity() if model else mu_field, -1.0)
        grad_p = fvm.gradient(p, p_opts["gradient"])
        fvm.eq_source(mom, -grad_p)
        if model:
            fvm.eq_source(mom, model.stress_remainder_divergence(U))
        if capture is not None:
            capture(it, dict(momentum=mom.ldu.copy()))
        rU = fvm.relative_residual(mom.ldu, U.v)
        fvm.eq_relax(mom, U_prev, settings.alpha_u)
        fvm.eq_scale(mom, settings.alpha_u)
        if capture is not None:
            capture(it, dict(momentum_relaxed=mom.ldu.copy()))
        aP = mom.ldu.diag.copy()
        rAU_v = V / aP
        U.v = _solve(mom.ldu.matrix(), mom.ldu.source)
        # Rhie-Chow (simple/main.cpp:71-79).
        grad_p = fvm.gradient(p, p_opts["gradient"])
        phiH = fvm.flux(U, mom_opts["interpolation"], mom_opts["gradient"])
        rAU = fvm.calculated(geo, rAU_v)
        # rAU*gradP is a calculated field: its traces are rAU's owner trace times
        # the boundary-corrected gradient trace (math.h fieldBinary, fvm_execution.cpp:213-237).
        g_trace = fvm.gradient_trace(p, grad_p)
        rAU_gradp = fvm.calculated(geo, rAU_v[:, None] * grad_p,
                                   trace_from=rAU_v[geo.owner][:, None] * g_trace)
        ifl = np.einsum("ij,ij->i", fvm.interpolate(rAU_gradp, p_opts["interpolation"], p_opts["gradient"]), geo.Sf)
        copts_i = p_opts.get("coefficientInterpolation") or p_opts["interpolation"]
        copts_g = p_opts.get("coefficientGradient") or p_opts["gradient"]
        nfl = fvm.interpolate(rAU, copts_i, copts_g) * fvm.normal_gradient(p, grad_p, p_opts["diffusion"]) * geo.area
        inn = geo.neighbour >= 0
        phiH = phiH.copy()
        phiH[inn] += ifl[inn]
        phiH[inn] -= nfl[inn]
        div_phiH = fvm.divergence_flux(geo, phiH)
        pP = fvm.Field(geo, np.zeros(nc), fvm.homogeneous_bcs(p_bcs))
        peq = None
        psystems = []
        for _ in range(pressure_solves):
            peq = fvm.Equation(pP, p_opts, {})
            fvm.eq_laplacian(peq, rAU, -1.0)
            fvm.eq_source(peq, -div_phiH)
            fvm.eq_reference_if_unanchored(peq, 0.0)
            psystems.append(peq.ldu.copy())
            pP.v = _solve(peq.ldu.matrix(), peq.ldu.source)
        if capture is not None:
            capture(it, dict(pressure=psystems, phiH=phiH.copy(), rAU=rAU_v.copy()))
        p.v = p.v + settings.alpha_p * pP.v
        pflux = fvm.eq_face_flux(peq, pP.v)
        U.v = U.v - rAU_v[:, None] * fvm.gradient(pP, p_opts["gradient"])
        phi = phiH + pflux
        turbulence_ok = True
        if model:
            t = model.solve_transport(U, phi)
            turbulence_ok = t["d"] <= model.c.tolerance and t["r"] <= model.c.tolerance
        dU = fvm.relative_change(U.v, U_prev)
        dP = fvm.relative_magnitude(pP.v, p.v)
        mass = fvm.flux_balance(geo, phi)
        conv = (turbulence_ok and rU <= settings.momentum_tolerance and dU <= settings.velocity_tolerance
                and dP <= settings.pressure_tolerance and mass["relative"] <= settings.mass_tolerance)
        state.history.append(dict(rU=rU, dU=dU, dP=dP, mass=mass["relative"]))
        state.U, state.p, state.phi, state.iterations = U.v, p.v, phi, it + 1
        if model:
            state.mut = model.mut_v
            for name, f in model.transported().items():
                setattr(state, name, f.v)
        if conv:
            state.converged = True
            break
    return state
