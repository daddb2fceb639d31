"""Wilcox-1988m k-omega and standard k-epsilon, restated from src/physics/RANS/k_omega.cpp,
k_epsilon.cpp and model.cpp.  TEST INFRASTRUCTURE ONLY.

Derived fields carry boundary traces exactly as the reference's calculated
fields do (include/babelsim/field.h:262-320, math.h:184-258): every pointwise
expression is applied to the cell values and to the boundary traces of its
operands, the traces of a field with boundary conditions being
Field::boundaryTrace (field.h:302-313).  The traces matter where the derived
fields meet faces: the viscosity and diffusivities in equ::laplacian and the
deviatoric stress in math::div(TensorField).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import fvm
from .simple import _solve


@dataclass
class KOmegaConstants:
    """Model constants and bounds (k_omega.cpp:31-41)."""
    beta_star: float = 0.09
    beta: float = 3.0 / 40.0
    gamma: float = 5.0 / 9.0
    sigma_k: float = 0.5
    sigma_omega: float = 0.5
    k_min: float = 1e-12
    omega_min: float = 1e-12
    viscosity_ratio_max: float = 1e5
    relaxation: float = 0.7
    tolerance: float = 1e-6


def strain_squared(G):
    """2 dev(symm(grad U)):dev(symm(grad U)) (k_omega.cpp:11-23); G rows = component gradients."""
    div = G[:, 0, 0] + G[:, 1, 1] + G[:, 2, 2]
    S = 0.5 * (G + np.transpose(G, (0, 2, 1)))
    for i in range(3):
        S[:, i, i] -= div / 3.0
    return 2.0 * np.sum(S * S, axis=(1, 2))


def _symmetric_tensor(G, n):
    """symmetricBoundaryValue(Tensor3) (include/babelsim/vector.h:107-116): 0.5 (G + R G R), R = I - 2 n n^T."""
    R = np.eye(3)[None] - 2.0 * n[:, :, None] * n[:, None, :]
    return 0.5 * (G + R @ G @ R)


def vector_gradient_trace(U: fvm.Field, G):
    """Boundary traces of a computed vector gradient (fvm_execution.cpp:240-262)."""
    geo = U.geo
    trace = np.zeros((geo.n_faces, 3, 3))
    bf = np.nonzero(geo.neighbour < 0)[0]
    o = geo.owner[bf]
    n = geo.normal[bf]
    d = geo.xf[bf] - geo.xc[o]
    dn = np.einsum("ij,ij->i", d, n)
    tang = d - dn[:, None] * n
    g = G[o].copy()
    types, values = fvm.face_condition(U, bf)
    sym = types == fvm.SYMMETRY
    if np.any(sym):
        g[sym] = _symmetric_tensor(g[sym], n[sym])
    rest = ~sym
    for c in range(3):
        gc = g[:, c, :]
        sn = np.where(types == fvm.FIXED_VALUE,
                      (values[:, c] - U.v[o, c] - np.einsum("ij,ij->i", gc, tang)) / np.where(dn != 0, dn, 1.0),
                      np.where(types == fvm.FIXED_GRADIENT, values[:, c], 0.0))
        upd = gc + (sn - np.einsum("ij,ij->i", gc, n))[:, None] * n
        g[rest, c, :] = upd[rest]
    trace[bf] = g
    return trace


def tensor_divergence(geo, T, T_trace, interpolation="linear"):
    """divergence(TensorField) (operators.cpp:1568-1591): each row reconstructed like a vector field."""
    if interpolation != "linear":
        raise NotImplementedError("the restatement covers linear reconstruction of the stress rows")
    out = np.zeros((geo.n_cells, 3))
    inn = np.nonzero(geo.neighbour >= 0)[0]
    bf = np.nonzero(geo.neighbour < 0)[0]
    w = geo.weight[inn]
    o, n = geo.owner[inn], geo.neighbour[inn]
    for c in range(3):
        fv = np.zeros((geo.n_faces, 3))
        fv[inn] = w[:, None] * T[o, c, :] + (1.0 - w)[:, None] * T[n, c, :]
        fv[bf] = T_trace[bf, c, :]
        contrib = np.einsum("ij,ij->i", fv, geo.Sf)
        col = np.zeros(geo.n_cells)
        np.add.at(col, geo.owner, contrib / geo.volume[geo.owner])
        np.add.at(col, geo.neighbour[inn], -contrib[inn] / geo.volume[geo.neighbour[inn]])
        out[:, c] = col
    return out


class KOmega:
    """KOmega (k_omega.cpp:25-160) on oracle fields."""

    def __init__(self, geo, k: fvm.Field, omega: fvm.Field, rho, mu, c: KOmegaConstants, k_opts, omega_opts,
                 momentum_opts, phi0):
        self.geo, self.k, self.omega, self.rho, self.mu, self.c = geo, k, omega, rho, mu, c
        self.k_opts, self.omega_opts, self.mom_opts = k_opts, omega_opts, momentum_opts
        self.bf = np.nonzero(geo.neighbour < 0)[0]
        nf = geo.n_faces
        # mut created as 0 then calculated: traces 0; muEffective created as mu then calculated (model.cpp:56-62)
        self.mut_v = np.zeros(geo.n_cells)
        self.mut_tr = np.zeros(nf)
        self.mueff_v = np.full(geo.n_cells, mu)
        self.mueff_tr = np.full(nf, mu)
        self.bound_transport_fields(phi0)
        self.update_viscosity()

    def _trace(self, f: fvm.Field):
        out = np.zeros(self.geo.n_faces)
        out[self.bf] = fvm.boundary_trace(f, self.bf)
        return out

    def bound_omega(self):
        k, w = self.k.v, self.omega.v
        lim = np.maximum(self.c.omega_min, self.rho * k / (self.c.viscosity_ratio_max * self.mu))
        self.omega.v = np.maximum(w, lim)

    def bound_transport_fields(self, phi):
        self.k.flux = np.array(phi, dtype=np.float64)
        self.omega.flux = np.array(phi, dtype=np.float64)
        self.k.v = np.maximum(self.k.v, self.c.k_min)
        self.bound_omega()

    def update_viscosity(self):
        """mut = rho k / max(omega, omegaMin); muEff = mu + mut (k_omega.cpp:153-156)."""
        wmin = self.c.omega_min
        self.mut_v = (self.rho * self.k.v) / np.maximum(self.omega.v, wmin)
        kt, wt = self._trace(self.k), self._trace(self.omega)
        self.mut_tr = np.zeros(self.geo.n_faces)
        self.mut_tr[self.bf] = (self.rho * kt[self.bf]) / np.maximum(wt[self.bf], wmin)
        self.mueff_v = self.mut_v + self.mu
        self.mueff_tr = self.mut_tr + self.mu

    def effective_viscosity(self):
        return fvm.Field(self.geo, self.mueff_v.copy(), None, trace=self.mueff_tr.copy())

    def transported(self):
        """The model's transported fields by state name (the second one is stored as omega)."""
        return {"k": self.k, "omega": self.omega}

    # Transient use (runPiso): time::history of each transported field, saved once per
    # physical step (saveOld), and equ::ddt(equation, rho, history) ahead of convection.
    time_method = None
    hist = None

    def set_transient(self, method):
        from .piso import History
        self.time_method = method
        self.hist = {name: History(f.copy()) for name, f in self.transported().items()}

    def save_old(self, dt):
        for name, f in self.transported().items():
            self.hist[name].save(f.copy(), dt)

    def _ddt(self, eq, name):
        if self.hist is not None:
            from .piso import eq_ddt
            eq_ddt(eq, self.rho, self.hist[name], self.time_method)

    def stress_remainder_divergence(self, U: fvm.Field):
        """math::div(muEff (grad(U)^T - 2/3 tr(grad U) I)) (model.cpp:65-69, operators.cpp:1568-1591)."""
        G = fvm.gradient(U, self.mom_opts["gradient"])
        Gt = vector_gradient_trace(U, G)

        def remainder(g, m):
            tr = g[:, 0, 0] + g[:, 1, 1] + g[:, 2, 2]
            iso = np.zeros_like(g)
            for i in range(3):
                iso[:, i, i] = tr
            return m[:, None, None] * (np.transpose(g, (0, 2, 1)) - (2.0 / 3.0) * iso)

        T = remainder(G, self.mueff_v)
        Tt = np.zeros_like(Gt)
        Tt[self.bf] = remainder(Gt[self.bf], self.mueff_tr[self.bf])
        return tensor_divergence(self.geo, T, Tt, self.mom_opts["interpolation"])

    def solve_transport(self, U: fvm.Field, phi):
        """KOmega::solveTransport (k_omega.cpp:65-125), steady (no time term)."""
        geo, c, rho, mu = self.geo, self.c, self.rho, self.mu
        prev_k, prev_w = self.k.v.copy(), self.omega.v.copy()
        U.flux = np.array(phi, dtype=np.float64)
        self.update_viscosity()
        G = fvm.gradient(U, self.mom_opts["gradient"])
        production = self.mut_v * strain_squared(G)
        k_diff = fvm.Field(geo, c.sigma_k * self.mut_v + mu, None, trace=c.sigma_k * self.mut_tr + mu)
        w_diff = fvm.Field(geo, c.sigma_omega * self.mut_v + mu, None, trace=c.sigma_omega * self.mut_tr + mu)
        w_destruction = (c.beta * rho) * self.omega.v
        w_production = ((c.gamma * production) * self.omega.v) / np.maximum(self.k.v, c.k_min)
        # omega first
        weq = fvm.Equation(self.omega, self.omega_opts, {})
        self._ddt(weq, "omega")
        fvm.eq_div(weq, phi, rho)
        fvm.eq_laplacian(weq, w_diff, -1.0)
        weq.ldu.diag = weq.ldu.diag + (1.0 * w_destruction) * geo.volume
        fvm.eq_source(weq, w_production)
        r_w = fvm.relative_residual(weq.ldu, self.omega.v)
        fvm.eq_relax(weq, prev_w, c.relaxation)
        self.omega.v = _solve(weq.ldu.matrix(), weq.ldu.source)
        self.bound_omega()
        # then k, with the new omega in its sink
        keq = fvm.Equation(self.k, self.k_opts, {})
        self._ddt(keq, "k")
        fvm.eq_div(keq, phi, rho)
        fvm.eq_laplacian(keq, k_diff, -1.0)
        keq.ldu.diag = keq.ldu.diag + (1.0 * ((c.beta_star * rho) * self.omega.v)) * geo.volume
        fvm.eq_source(keq, production)
        r_k = fvm.relative_residual(keq.ldu, self.k.v)
        fvm.eq_relax(keq, prev_k, c.relaxation)
        self.k.v = _solve(keq.ldu.matrix(), keq.ldu.source)
        self.bound_transport_fields(phi)
        self.update_viscosity()
        return dict(d=max(fvm.relative_change(self.omega.v, prev_w), fvm.relative_change(self.k.v, prev_k)),
                    r=max(r_w, r_k))


@dataclass
class KEpsilonConstants:
    """Model constants and bounds (k_epsilon.cpp:31-39)."""
    c_mu: float = 0.09
    c1: float = 1.44
    c2: float = 1.92
    sigma_k: float = 1.0
    sigma_epsilon: float = 1.3
    k_min: float = 1e-12
    epsilon_min: float = 1e-12
    relaxation: float = 0.7
    tolerance: float = 1e-6


class KEpsilon(KOmega):
    """KEpsilon (k_epsilon.cpp:25-128) on oracle fields: k first, then epsilon, one frozen closure state."""

    def __init__(self, geo, k: fvm.Field, epsilon: fvm.Field, rho, mu, c: KEpsilonConstants, k_opts, eps_opts,
                 momentum_opts, phi0):
        self.geo, self.k, self.eps, self.rho, self.mu, self.c = geo, k, epsilon, rho, mu, c
        self.k_opts, self.eps_opts, self.mom_opts = k_opts, eps_opts, momentum_opts
        self.bf = np.nonzero(geo.neighbour < 0)[0]
        nf = geo.n_faces
        self.mut_v = np.zeros(geo.n_cells)
        self.mut_tr = np.zeros(nf)
        self.mueff_v = np.full(geo.n_cells, mu)
        self.mueff_tr = np.full(nf, mu)
        self.bound_transport_fields(phi0)
        self.update_viscosity()

    @property
    def omega(self):  # the second transported field, for callers that read both
        return self.eps

    def bound_transport_fields(self, phi):
        self.k.flux = np.array(phi, dtype=np.float64)
        self.eps.flux = np.array(phi, dtype=np.float64)
        self.k.v = np.maximum(self.k.v, self.c.k_min)
        self.eps.v = np.maximum(self.eps.v, self.c.epsilon_min)

    def update_viscosity(self):
        """mut = Cmu rho k k / max(epsilon, epsilonMin); muEff = mu + mut (k_epsilon.cpp:122-125)."""
        emin = self.c.epsilon_min
        cr = self.c.c_mu * self.rho
        self.mut_v = ((cr * self.k.v) * self.k.v) / np.maximum(self.eps.v, emin)
        kt, et = self._trace(self.k), self._trace(self.eps)
        self.mut_tr = np.zeros(self.geo.n_faces)
        b = self.bf
        self.mut_tr[b] = ((cr * kt[b]) * kt[b]) / np.maximum(et[b], emin)
        self.mueff_v = self.mut_v + self.mu
        self.mueff_tr = self.mut_tr + self.mu

    def solve_transport(self, U: fvm.Field, phi):
        """KEpsilon::solveTransport (k_epsilon.cpp:62-111), steady."""
        geo, c, rho, mu = self.geo, self.c, self.rho, self.mu
        prev_k, prev_e = self.k.v.copy(), self.eps.v.copy()
        U.flux = np.array(phi, dtype=np.float64)
        self.update_viscosity()
        G = fvm.gradient(U, self.mom_opts["gradient"])
        production = self.mut_v * strain_squared(G)
        k_diff = fvm.Field(geo, (1.0 / c.sigma_k) * self.mut_v + mu, None, trace=(1.0 / c.sigma_k) * self.mut_tr + mu)
        e_diff = fvm.Field(geo, (1.0 / c.sigma_epsilon) * self.mut_v + mu, None,
                           trace=(1.0 / c.sigma_epsilon) * self.mut_tr + mu)
        eok = self.eps.v / np.maximum(self.k.v, c.k_min)
        k_destruction = rho * eok
        e_destruction = (c.c2 * rho) * eok
        e_production = (c.c1 * production) * eok
        keq = fvm.Equation(self.k, self.k_opts, {})
        self._ddt(keq, "k")
        fvm.eq_div(keq, phi, rho)
        fvm.eq_laplacian(keq, k_diff, -1.0)
        keq.ldu.diag = keq.ldu.diag + (1.0 * k_destruction) * geo.volume
        fvm.eq_source(keq, production)
        r_k = fvm.relative_residual(keq.ldu, self.k.v)
        fvm.eq_relax(keq, prev_k, c.relaxation)
        self.k.v = _solve(keq.ldu.matrix(), keq.ldu.source)
        eeq = fvm.Equation(self.eps, self.eps_opts, {})
        self._ddt(eeq, "omega")
        fvm.eq_div(eeq, phi, rho)
        fvm.eq_laplacian(eeq, e_diff, -1.0)
        eeq.ldu.diag = eeq.ldu.diag + (1.0 * e_destruction) * geo.volume
        fvm.eq_source(eeq, e_production)
        r_e = fvm.relative_residual(eeq.ldu, self.eps.v)
        fvm.eq_relax(eeq, prev_e, c.relaxation)
        self.eps.v = _solve(eeq.ldu.matrix(), eeq.ldu.source)
        self.bound_transport_fields(phi)
        self.update_viscosity()
        return dict(d=max(fvm.relative_change(self.k.v, prev_k), fvm.relative_change(self.eps.v, prev_e)),
                    r=max(r_k, r_e))


@dataclass
class SpalartAllmarasConstants:
    """Model constants and bounds (spalart_allmaras.cpp:31-45); cw1 defaults to cb1/kappa^2 + (1 + cb2)/sigma."""
    cb1: float = 0.1355
    cb2: float = 0.622
    sigma: float = 2.0 / 3.0
    kappa: float = 0.41
    cw2: float = 0.3
    cw3: float = 2.0
    cv1: float = 7.1
    ct3: float = 1.2
    ct4: float = 0.5
    cw1: float | None = None
    nu_tilda_min: float = 1e-14
    wall_distance_min: float = 1e-12
    relaxation: float = 0.7
    tolerance: float = 1e-6

    def __post_init__(self):
        if self.cw1 is None:
            self.cw1 = self.cb1 / (self.kappa * self.kappa) + (1.0 + self.cb2) / self.sigma


def vorticity_magnitude(G):
    """sqrt(2 sum_ij (0.5 (G_ij - G_ji))^2) per cell, summed row by row (spalart_allmaras.cpp:10-19)."""
    s = np.zeros(G.shape[0])
    for i in range(3):
        for j in range(3):
            rot = 0.5 * (G[:, i, j] - G[:, j, i])
            s = s + rot * rot
    return np.sqrt(2.0 * s)


class SpalartAllmaras(KOmega):
    """SpalartAllmaras (spalart_allmaras.cpp:23-154) on oracle fields: positive-variable SA with ft2 and
    without the trip term; the wall distance is a given cell field."""

    def __init__(self, geo, nu_tilda: fvm.Field, wall_distance, rho, mu, c: SpalartAllmarasConstants, nt_opts,
                 momentum_opts, phi0):
        self.geo, self.nt, self.rho, self.mu, self.c = geo, nu_tilda, rho, mu, c
        self.wall_distance = np.asarray(wall_distance, dtype=np.float64)
        self.nt_opts, self.mom_opts = nt_opts, momentum_opts
        self.bf = np.nonzero(geo.neighbour < 0)[0]
        nf = geo.n_faces
        self.mut_v = np.zeros(geo.n_cells)
        self.mut_tr = np.zeros(nf)
        self.mueff_v = np.full(geo.n_cells, mu)
        self.mueff_tr = np.full(nf, mu)
        self.bound_transport_fields(phi0)
        self.update_viscosity()

    def transported(self):
        return {"nuTilda": self.nt}

    def _fv1(self, chi):
        chi3 = (chi * chi) * chi
        cv = self.c.cv1
        return chi3 / (chi3 + (cv * cv) * cv)

    def bound_transport_fields(self, phi):
        self.nt.flux = np.array(phi, dtype=np.float64)
        self.nt.v = np.maximum(self.nt.v, self.c.nu_tilda_min)

    def update_viscosity(self):
        """mut = rho nuTilda fv1(nuTilda / nu); muEff = mu + mut, with calculated traces (:137-140)."""
        nu = self.mu / self.rho
        self.mut_v = (self.rho * self.nt.v) * self._fv1(self.nt.v / nu)
        tr = self._trace(self.nt)
        b = self.bf
        self.mut_tr = np.zeros(self.geo.n_faces)
        self.mut_tr[b] = (self.rho * tr[b]) * self._fv1(tr[b] / nu)
        self.mueff_v = self.mut_v + self.mu
        self.mueff_tr = self.mut_tr + self.mu

    def solve_transport(self, U: fvm.Field, phi):
        """SpalartAllmaras::solveTransport (:65-122), steady (the time term is absent)."""
        geo, c, rho, mu = self.geo, self.c, self.rho, self.mu
        prev = self.nt.v.copy()
        U.flux = np.array(phi, dtype=np.float64)
        nt = self.nt.v
        nu = mu / rho
        chi = nt / nu
        fv1 = self._fv1(chi)
        fv2 = 1.0 - chi / (1.0 + chi * fv1)
        ft2 = c.ct3 * np.exp(((-c.ct4) * chi) * chi)
        distance = np.maximum(self.wall_distance, c.wall_distance_min)
        inv_d2 = 1.0 / (distance * distance)
        k2 = c.kappa * c.kappa
        rotation = vorticity_magnitude(fvm.gradient(U, self.mom_opts["gradient"]))
        mod_rot = np.maximum(rotation + ((nt * fv2) * inv_d2) / k2, 1e-30)
        r = np.clip((nt * inv_d2) / (k2 * mod_rot), 0.0, 10.0)
        g = r + c.cw2 * (r ** 6.0 - r)
        cw3_6 = c.cw3 ** 6.0
        fw = g * ((1.0 + cw3_6) / (g ** 6.0 + cw3_6)) ** (1.0 / 6.0)
        production = (c.cb1 * (1.0 - ft2)) * mod_rot
        destruction = ((c.cw1 * fw - (c.cb1 / k2) * ft2) * nt) * inv_d2
        net = production - destruction
        implicit = rho * np.maximum(-net, 0.0)
        gnt = fvm.gradient(self.nt, self.nt_opts["gradient"])
        grad_source = ((rho * c.cb2) / c.sigma) * np.einsum("ij,ij->i", gnt, gnt)
        explicit = (rho * np.maximum(net, 0.0)) * nt + grad_source
        tr = self._trace(self.nt)
        diff = fvm.Field(geo, (mu + rho * nt) / c.sigma, None, trace=(mu + rho * tr) / c.sigma)
        eq = fvm.Equation(self.nt, self.nt_opts, {})
        self._ddt(eq, "nuTilda")
        fvm.eq_div(eq, phi, rho)
        fvm.eq_laplacian(eq, diff, -1.0)
        eq.ldu.diag = eq.ldu.diag + (1.0 * implicit) * geo.volume
        fvm.eq_source(eq, explicit)
        res = fvm.relative_residual(eq.ldu, self.nt.v)
        fvm.eq_relax(eq, prev, c.relaxation)
        self.nt.v = _solve(eq.ldu.matrix(), eq.ldu.source)
        self.bound_transport_fields(phi)
        self.update_viscosity()
        return dict(d=fvm.relative_change(self.nt.v, prev), r=res)
