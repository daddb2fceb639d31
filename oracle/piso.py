"""Transient PISO, restated from src/physics/piso/main.cpp:60-301.  TEST INFRASTRUCTURE ONLY.

Laminar, constant density and viscosity, no potential-flow initialisation.
Linear systems are solved directly (sparse LU), which stands in for the
reference's Krylov solves converged to their tolerance.  Time levels follow
time::History (include/babelsim/history.h) and TimeStepper::advance
(src/io/case.cpp:391-403); the transient term follows equ::ddt's variable-step
BDF2 (src/discretization/procedural_equation.cpp:198-223).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import fvm
from .simple import _solve


@dataclass
class PisoSettings:
    """The PISO controls of piso/main.cpp:76-99 plus the per-equation options."""
    rho: float = 1.0
    mu: float = 0.01
    alpha_u: float = 1.0
    max_iterations: int = 1
    correctors: int = 2
    max_correctors: int | None = None
    coupling_tolerance: float = float(np.finfo(np.float64).max)
    non_orthogonal_corrections: int = 1
    mass_tolerance: float = 1e-8
    velocity_tolerance: float = 1e-7
    momentum_tolerance: float = 1e-6
    pressure_tolerance: float = 1e-6
    time: str = "bdf2"
    start_time: float = 0.0
    end_time: float = 1.0
    delta_t: float = 1e-3
    initialize_potential_flow: bool = False
    initial_non_orthogonal_corrections: int | None = None
    turbulence_coupling: str = "iterated"
    turbulence_max_iterations: int = 1000
    turbulence_correctors: int | None = None
    momentum: dict = field(default_factory=lambda: dict(
        interpolation="linear", gradient="greenGauss", convection="upwind", diffusion="orthogonal"))
    pressure: dict = field(default_factory=lambda: dict(
        interpolation="linear", gradient="greenGauss", convection="upwind", diffusion="orthogonal"))


class History:
    """time::History<T> (include/babelsim/history.h:5-22): previous/older levels and their steps."""

    def __init__(self, f):
        self.previous = f
        self.older = f
        self.dt = 0.0
        self.previous_dt = 0.0
        self.levels = 0

    def save(self, f, dt):
        self.older = self.previous
        self.previous = f
        self.previous_dt = self.dt
        self.dt = dt
        self.levels += 1


def time_weights(method, dt, older_dt):
    """timeTerm coefficients (procedural_equation.cpp:205-214): a0 diag, a1 previous, a2 older."""
    a0 = a1 = 1.0 / dt
    a2 = 0.0
    if method == "bdf2":
        if older_dt == 0.0:
            older_dt = dt
        r = dt / older_dt
        a0 = (1 + 2 * r) / ((1 + r) * dt)
        a1 = (1 + r) / dt
        a2 = -r * r / ((1 + r) * dt)
    return a0, a1, a2


def eq_ddt(eq: fvm.Equation, capacity, hist: History, configured):
    """equ::ddt(Equation, capacity, History) (procedural_equation.cpp:225-231, 198-223)."""
    method = "euler" if configured == "bdf2" and hist.levels < 2 else configured
    a0, a1, a2 = time_weights(method, hist.dt, hist.previous_dt)
    geo = eq.x.geo
    w = capacity * geo.volume
    q = eq.ldu
    q.diag = q.diag + w * a0
    prev = hist.previous.v
    older = hist.older.v
    if prev.ndim == 2:
        q.source = q.source + (w * a1)[:, None] * prev
        if a2 != 0.0:
            q.source = q.source + (w * a2)[:, None] * older
    else:
        q.source = q.source + (w * a1) * prev
        if a2 != 0.0:
            q.source = q.source + (w * a2) * older


def temporal_flux_correction(U_old: History, phi_old: History, method, opts):
    """temporalFluxCorrection (piso/main.cpp:19-55): interior faces only."""
    dt = U_old.dt
    w_prev, w_older = 1.0 / dt, 0.0
    if method == "bdf2" and U_old.levels >= 2:
        ratio = dt / U_old.previous_dt
        w_prev = (1.0 + ratio) / dt
        w_older = -ratio * ratio / ((1.0 + ratio) * dt)
    prev_U = U_old.previous.copy()
    mismatch = phi_old.previous - fvm.flux(prev_U, opts["interpolation"], opts["gradient"])
    correction = w_prev * mismatch
    if w_older != 0.0:
        older_U = U_old.older.copy()
        correction = correction + w_older * (phi_old.older - fvm.flux(older_U, opts["interpolation"], opts["gradient"]))
    f = phi_old.previous
    coupling = np.where(mismatch == 0.0, 1.0,
                        np.where(f == 0.0, 0.0, np.maximum(0.0, 1.0 - np.abs(mismatch) / np.where(f == 0.0, 1.0, np.abs(f)))))
    geo = U_old.previous.geo
    out = np.zeros(geo.n_faces)
    inn = geo.neighbour >= 0
    out[inn] = (coupling * correction)[inn]
    return out


def advance_time(value, step, start, end, dt):
    """TimeStepper::advance (src/io/case.cpp:391-403): next level and its step."""
    eps = np.finfo(np.float64).eps
    tol = 32 * eps * max(abs(start), abs(end), dt)
    nxt = float(np.longdouble(start) + np.longdouble(step + 1) * np.longdouble(dt))
    if nxt >= end - tol:
        nxt = end
    return nxt, nxt - value


@dataclass
class PisoState:
    U: np.ndarray
    p: np.ndarray
    phi: np.ndarray
    time: float = 0.0
    steps: int = 0
    status: str = "running"
    history: list = field(default_factory=list)


def run_piso(geo, U_bcs, p_bcs, s: PisoSettings, U0=None, p0=None, steps=None, turbulence=None) -> PisoState:
    """runPiso (piso/main.cpp:60-301) for `steps` time steps (all, to end_time, when None).
    ``turbulence(geo, phi)`` builds an eddy-viscosity model (oracle.rans), created like rans::load
    before phi = flux(U), i.e. with a zero face flux."""
    nc = geo.n_cells
    U = fvm.Field(geo, np.zeros((nc, 3)) if U0 is None else U0, U_bcs)
    p = fvm.Field(geo, np.zeros(nc) if p0 is None else p0, p_bcs)
    m_opts, p_opts = dict(s.momentum), dict(s.pressure)
    pressure_solves = 1 if p_opts["diffusion"] == "orthogonal" else s.non_orthogonal_corrections + 1
    max_correctors = s.correctors if s.max_correctors is None else s.max_correctors
    V = geo.volume
    mu_field = fvm.Field(geo, np.full(nc, s.mu), [(fvm.ZERO_GRADIENT, 0.0)] * len(U_bcs))
    model = turbulence(geo, np.zeros(geo.n_faces)) if turbulence is not None else None
    segregated = s.turbulence_coupling == "segregated"
    if model is not None:
        model.set_transient(s.time)
    t_corrections = s.turbulence_correctors or (
        s.turbulence_max_iterations if model is not None and s.max_iterations == 1 and not segregated else 1)
    phi = fvm.flux(U, p_opts["interpolation"], p_opts["gradient"])
    if s.initialize_potential_flow:
        # a conservative initial flux from a potential solve (piso/main.cpp:123-146)
        init_corr = s.non_orthogonal_corrections if s.initial_non_orthogonal_corrections is None \
            else s.initial_non_orthogonal_corrections
        n_solves = 1 if p_opts["diffusion"] == "orthogonal" else init_corr + 1
        pP = fvm.Field(geo, np.zeros(nc), fvm.homogeneous_bcs(p_bcs))
        imbalance = fvm.divergence_flux(geo, phi)
        peq = None
        for _ in range(n_solves):
            peq = fvm.Equation(pP, p_opts, {})
            fvm.eq_laplacian(peq, 1.0, -1.0)
            fvm.eq_source(peq, -imbalance)
            fvm.eq_reference_if_unanchored(peq, 0.0)
            pP.v = _solve(peq.ldu.matrix(), peq.ldu.source)
        U.v = U.v - fvm.gradient(pP, p_opts["gradient"])
        phi = phi + fvm.eq_face_flux(peq, pP.v)
        U.flux = phi.copy()
    U_old = History(U.copy())
    phi_old = History(phi.copy())
    state = PisoState(U.v, p.v, phi, s.start_time)
    t, step = s.start_time, 0
    copt_i = p_opts.get("coefficientInterpolation") or p_opts["interpolation"]
    copt_g = p_opts.get("coefficientGradient") or p_opts["gradient"]
    inn = geo.neighbour >= 0
    while t < s.end_time and (steps is None or step < steps):
        t, dt = advance_time(t, step, s.start_time, s.end_time, s.delta_t)
        step += 1
        U_old.save(U.copy(), dt)
        phi_old.save(phi.copy(), dt)
        if model is not None:
            model.save_old(dt)
        temporal = s.rho * temporal_flux_correction(U_old, phi_old, s.time, p_opts)
        converged = False
        for _ in range(s.max_iterations):
            U_prev = U.v.copy()
            mom = fvm.Equation(U, m_opts, {})
            eq_ddt(mom, s.rho, U_old, s.time)
            fvm.eq_div(mom, phi, s.rho)
            fvm.eq_laplacian(mom, model.effective_viscosity() if model is not None else mu_field, -1.0)
            grad_p = fvm.gradient(p, p_opts["gradient"])
            fvm.eq_source(mom, -grad_p)
            if model is not None:
                fvm.eq_source(mom, model.stress_remainder_divergence(U))
            rU = fvm.relative_residual(mom.ldu, U.v)
            fvm.eq_relax(mom, U_prev, s.alpha_u)
            aP = mom.ldu.diag.copy()
            rAU_v = V / aP
            inv_aP = 1.0 / aP
            rAU = fvm.calculated(geo, rAU_v)
            rAUf = fvm.interpolate(rAU, copt_i, copt_g)
            npr = mom.ldu.source + V[:, None] * grad_p
            U.v = _solve(mom.ldu.matrix(), mom.ldu.source)
            dP = coupling = 0.0
            used = 0
            for corrector in range(max_correctors):
                HbyA = fvm.Field(geo, inv_aP[:, None] * (npr - mom.ldu.apply(U.v) + aP[:, None] * U.v), U_bcs,
                                 flux=phi)
                p_prev = p.v.copy()
                phiH = fvm.flux(HbyA, p_opts["interpolation"], p_opts["gradient"]).copy()
                phiH[inn] += (rAUf * temporal)[inn]
                imbalance = fvm.divergence_flux(geo, phiH)
                peq = None
                for _ in range(pressure_solves):
                    peq = fvm.Equation(p, p_opts, {})
                    fvm.eq_laplacian(peq, rAUf, -1.0)
                    fvm.eq_source(peq, -imbalance)
                    fvm.eq_reference_if_unanchored(peq, 0.0)
                    p.v = _solve(peq.ldu.matrix(), peq.ldu.source)
                phi = phiH + fvm.eq_face_flux(peq, p.v)
                gp = fvm.gradient(p, p_opts["gradient"])
                U.v = HbyA.v - rAU_v[:, None] * gp
                U.flux = phi.copy()
                dP = max(dP, fvm.relative_magnitude(p.v - p_prev, p.v))
                action = mom.ldu.apply(U.v)
                psrc = V[:, None] * gp
                defect = npr - action - psrc
                n0, n1, n2, n3 = (float(np.sqrt(np.sum(a * a))) for a in (npr, action, psrc, defect))
                scale = n0 + n1 + n2
                coupling = n3 / scale if scale > 0.0 else n3
                used = corrector + 1
                if used >= s.correctors and coupling <= s.coupling_tolerance:
                    break
            t_ok, t_corr, dT, rT = True, 0, 0.0, 0.0
            if model is not None:
                # turbulence correctors at this time level (piso/main.cpp:239-254)
                for _ in range(t_corrections):
                    r = model.solve_transport(U, phi)
                    dT, rT = r["d"], r["r"]
                    t_corr += 1
                    t_ok = dT <= model.c.tolerance and rT <= model.c.tolerance
                    if t_ok:
                        break
            dU = fvm.relative_change(U.v, U_prev)
            mass = fvm.flux_balance(geo, phi)["relative"]
            accepted = mass <= s.mass_tolerance and coupling <= s.coupling_tolerance
            settled = (rU <= s.momentum_tolerance and dU <= s.velocity_tolerance and dP <= s.pressure_tolerance
                       and t_ok)
            converged = accepted and ((segregated or t_ok) if s.max_iterations == 1 else settled)
            state.history.append(dict(step=step, rU=rU, dU=dU, dP=dP, mass=mass, coupling=coupling, correctors=used,
                                      dTurb=dT, rTurb=rT, turbulence_corrections=t_corr))
            if not accepted:
                state.status = "notConverged"
                break
            if converged:
                break
        state.U, state.p, state.phi, state.time, state.steps = U.v, p.v, phi, t, step
        if model is not None:
            state.mut = model.mut_v
            for name, f in model.transported().items():
                setattr(state, name, f.v)
        if not converged:
            state.status = "notConverged"
            return state
    state.status = "completed" if t >= s.end_time else "running"
    return state

