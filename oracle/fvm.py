"""Finite-volume operators and LDU assembly, restated in numpy.  TEST INFRASTRUCTURE ONLY.

Every function cites the reference code it follows (paths inside the BabelSim
project).  Face loops become array operations over faces; accumulation into
cells uses ``np.add.at`` (unbuffered, so repeated owner/neighbour indices add
up exactly like the reference's sequential loop, up to summation order).

Boundary-condition codes follow ``BoundaryType`` (include/babelsim/field.h:23-32).
"""
from __future__ import annotations

import numpy as np

FIXED_VALUE, FIXED_GRADIENT, ZERO_GRADIENT, INLET_OUTLET, SYMMETRY = 0, 1, 2, 3, 4
BC_NAMES = {"fixedValue": FIXED_VALUE, "fixedGradient": FIXED_GRADIENT, "zeroGradient": ZERO_GRADIENT,
            "inletOutlet": INLET_OUTLET, "symmetry": SYMMETRY}
EPS = np.finfo(np.float64).eps


class Field:
    """Cell field with per-patch constraints, or a calculated field with per-face traces.

    Mirrors Field<T> (include/babelsim/field.h:57-374): ``bcs`` holds one
    (type, value) per patch; a calculated field instead carries ``trace`` (one
    value per face, meaningful on boundary faces).  ``flux`` is the saved
    boundary-flux context used by inletOutlet (field.h:274-299).
    """

    def __init__(self, geo, values, bcs=None, trace=None, flux=None):
        self.geo = geo
        self.v = np.array(values, dtype=np.float64)
        self.bcs = bcs
        self.trace = trace
        self.flux = None if flux is None else np.array(flux, dtype=np.float64)

    @property
    def vector(self):
        return self.v.ndim == 2

    def copy(self):
        return Field(self.geo, self.v.copy(), self.bcs, None if self.trace is None else self.trace.copy(),
                     self.flux)

    def with_values(self, values):
        return Field(self.geo, values, self.bcs, self.trace, self.flux)


def calculated(geo, values, trace_from=None):
    """A derived field whose boundary traces are the owner values (useCalculatedBoundary on default BCs)."""
    values = np.asarray(values, dtype=np.float64)
    trace = values[geo.owner] if trace_from is None else trace_from
    return Field(geo, values, None, trace)


def _bfaces(geo):
    return np.nonzero(geo.neighbour < 0)[0]


def face_condition(field: Field, faces, outward_flux=None):
    """Per-face (type, value) for boundary faces: Field::faceCondition (field.h:285-301)."""
    geo = field.geo
    n = len(faces)
    vshape = (n, 3) if field.vector else (n,)
    if field.bcs is None:
        return np.full(n, FIXED_VALUE), field.trace[faces].copy()
    types = np.empty(n, dtype=np.int64)
    values = np.zeros(vshape)
    patches = geo.patch[faces]
    for p, (t, val) in enumerate(field.bcs):
        m = patches == p
        types[m] = t
        values[m] = val
    io = types == INLET_OUTLET
    if np.any(io):
        if outward_flux is None:
            if field.flux is None:
                raise ValueError("inletOutlet requires a boundary flux context")
            fl = field.flux[faces]
        else:
            fl = np.broadcast_to(np.asarray(outward_flux, dtype=np.float64), (n,))
        inflow = io & (fl < 0.0)
        outflow = io & ~(fl < 0.0)
        types[inflow] = FIXED_VALUE
        types[outflow] = ZERO_GRADIENT
        values[outflow] = 0.0
    return types, values


def boundary_trace(field: Field, faces, outward_flux=None):
    """Field::boundaryTrace (field.h:302-313)."""
    geo = field.geo
    types, values = face_condition(field, faces, outward_flux)
    own = field.v[geo.owner[faces]]
    out = own.copy()
    fv = types == FIXED_VALUE
    out[fv] = values[fv]
    fg = types == FIXED_GRADIENT
    if np.any(fg):
        d = np.einsum("ij,ij->i", geo.xf[faces] - geo.xc[geo.owner[faces]], geo.normal[faces])
        out[fg] = own[fg] + (d[fg][:, None] * values[fg] if field.vector else d[fg] * values[fg])
    sy = types == SYMMETRY
    if np.any(sy) and field.vector:
        n = geo.normal[faces][sy]
        o = own[sy]
        out[sy] = o - np.einsum("ij,ij->i", o, n)[:, None] * n
    return out


def _w(geo, faces):
    return geo.weight[faces]


def interpolate_linear(field: Field, outward_flux=None):
    """interpolatedFaceValue over all faces (operators.cpp:231-237, 34-43)."""
    geo = field.geo
    shape = (geo.n_faces, 3) if field.vector else (geo.n_faces,)
    out = np.zeros(shape)
    inn = np.nonzero(geo.neighbour >= 0)[0]
    w = geo.weight[inn]
    o, n = geo.owner[inn], geo.neighbour[inn]
    if field.vector:
        out[inn] = w[:, None] * field.v[o] + (1.0 - w)[:, None] * field.v[n]
    else:
        out[inn] = w * field.v[o] + (1.0 - w) * field.v[n]
    bf = _bfaces(geo)
    out[bf] = boundary_trace(field, bf, None if outward_flux is None else outward_flux[bf])
    return out


def _face_grad(geo, grad, faces):
    w = geo.weight[faces]
    o, n = geo.owner[faces], geo.neighbour[faces]
    if grad.ndim == 2:
        return w[:, None] * grad[o] + (1.0 - w)[:, None] * grad[n]
    return w[:, None, None] * grad[o] + (1.0 - w)[:, None, None] * grad[n]


def corrected_interior(field: Field, grad, faces):
    """correctedInternalFaceValue (operators.cpp:45-81)."""
    geo = field.geo
    w = geo.weight[faces]
    o, n = geo.owner[faces], geo.neighbour[faces]
    fg = _face_grad(geo, grad, faces)
    if field.vector:
        lin = w[:, None] * field.v[o] + (1.0 - w)[:, None] * field.v[n]
        return lin + np.einsum("fcj,fj->fc", fg, geo.skew[faces])
    lin = w * field.v[o] + (1.0 - w) * field.v[n]
    return lin + np.einsum("fj,fj->f", fg, geo.skew[faces])


def reconstructed_boundary(field: Field, grad, faces, outward_flux=None):
    """reconstructedBoundaryValue (operators.cpp:110-164)."""
    geo = field.geo
    types, values = face_condition(field, faces, outward_flux)
    o = geo.owner[faces]
    nrm = geo.normal[faces]
    off = geo.xf[faces] - geo.xc[o]
    if field.vector:
        out = field.v[o].copy()
        for c in range(3):
            pres = np.where(types == FIXED_GRADIENT, values[:, c], 0.0)
            g = grad[o][:, c, :]
            gc = g + (pres - np.einsum("ij,ij->i", g, nrm))[:, None] * nrm
            out[:, c] += np.einsum("ij,ij->i", gc, off)
        sy = types == SYMMETRY
        out[sy] -= np.einsum("ij,ij->i", out[sy], nrm[sy])[:, None] * nrm[sy]
    else:
        pres = np.where(types == FIXED_GRADIENT, values, 0.0)
        g = grad[o]
        gc = g + (pres - np.einsum("ij,ij->i", g, nrm))[:, None] * nrm
        out = field.v[o] + np.einsum("ij,ij->i", gc, off)
    fv = types == FIXED_VALUE
    out[fv] = values[fv]
    return out


def corrected_face_values(field: Field, grad, outward_flux=None):
    """correctedFaceValue over all faces (operators.cpp:166-186)."""
    geo = field.geo
    shape = (geo.n_faces, 3) if field.vector else (geo.n_faces,)
    out = np.zeros(shape)
    inn = np.nonzero(geo.neighbour >= 0)[0]
    out[inn] = corrected_interior(field, grad, inn)
    bf = _bfaces(geo)
    out[bf] = reconstructed_boundary(field, grad, bf, None if outward_flux is None else outward_flux[bf])
    return out


def _gauss_sum(geo, face_values):
    """sum_f +/- phi_f Sf / V (the accumulation loops of operators.cpp:275-316)."""
    nc = geo.n_cells
    inn = geo.neighbour >= 0
    if face_values.ndim == 1:
        contrib = face_values[:, None] * geo.Sf
        out = np.zeros((nc, 3))
        np.add.at(out, geo.owner, contrib / geo.volume[geo.owner][:, None])
        np.add.at(out, geo.neighbour[inn], -contrib[inn] / geo.volume[geo.neighbour[inn]][:, None])
    else:
        contrib = face_values[:, :, None] * geo.Sf[:, None, :]
        out = np.zeros((nc, 3, 3))
        np.add.at(out, geo.owner, contrib / geo.volume[geo.owner][:, None, None])
        np.add.at(out, geo.neighbour[inn], -contrib[inn] / geo.volume[geo.neighbour[inn]][:, None, None])
    return out


def gradient_green_gauss(field: Field):
    """greenGaussGradient scalar/vector (operators.cpp:275-316, 365-405)."""
    geo = field.geo
    g = _gauss_sum(geo, interpolate_linear(field))
    if geo.orthogonal:
        return g
    return _gauss_sum(geo, corrected_face_values(field, g))


def gradient_trace(field: Field, g):
    """Boundary traces of a computed scalar gradient (fvm_execution.cpp:213-237)."""
    geo = field.geo
    trace = np.zeros((geo.n_faces, 3))
    bf = _bfaces(geo)
    o = geo.owner[bf]
    n = geo.normal[bf]
    d = geo.xf[bf] - geo.xc[o]
    gb = g[o].copy()
    types, values = face_condition(field, bf)
    dn = np.einsum("ij,ij->i", d, n)
    tang = d - dn[:, None] * n
    sn = np.where(types == FIXED_VALUE,
                  (values - field.v[o] - np.einsum("ij,ij->i", gb, tang)) / np.where(dn != 0, dn, 1.0),
                  np.where(types == FIXED_GRADIENT, values, 0.0))
    gb += (sn - np.einsum("ij,ij->i", gb, n))[:, None] * n
    trace[bf] = gb
    return trace


def _boundary_normal_distance(geo, faces):
    """boundaryNormalDistance (src/internal/boundary_evaluation.h:7-13)."""
    return np.einsum("ij,ij->i", geo.xf[faces] - geo.xc[geo.owner[faces]], geo.normal[faces])


def gradient_least_squares(field: Field):
    """leastSquaresGradient scalar/vector (operators.cpp:318-363, 407-458)."""
    geo = field.geo
    nc = geo.n_cells
    inn = np.nonzero(geo.neighbour >= 0)[0]
    bf = _bfaces(geo)
    M = np.zeros((nc, 3, 3))
    R = np.zeros((nc, 3, 3)) if field.vector else np.zeros((nc, 3))
    o, n = geo.owner[inn], geo.neighbour[inn]
    for cell, other in ((o, n), (n, o)):
        d = geo.xc[other] - geo.xc[cell]
        diff = field.v[other] - field.v[cell]
        wgt = 1.0 / np.einsum("ij,ij->i", d, d)
        np.add.at(M, cell, wgt[:, None, None] * d[:, :, None] * d[:, None, :])
        if field.vector:
            np.add.at(R, cell, wgt[:, None, None] * d[:, :, None] * diff[:, None, :])
        else:
            np.add.at(R, cell, wgt[:, None] * d * diff[:, None])
    ob = geo.owner[bf]
    types, _ = face_condition(field, bf)
    off = geo.xf[bf] - geo.xc[ob]
    dist = _boundary_normal_distance(geo, bf)
    d = np.where((types == FIXED_VALUE)[:, None], 2.0 * off, 2.0 * dist[:, None] * geo.normal[bf])
    diff = 2.0 * (boundary_trace(field, bf) - field.v[ob])
    wgt = 1.0 / np.einsum("ij,ij->i", d, d)
    np.add.at(M, ob, wgt[:, None, None] * d[:, :, None] * d[:, None, :])
    if field.vector:
        np.add.at(R, ob, wgt[:, None, None] * d[:, :, None] * diff[:, None, :])
        sol = np.linalg.solve(M, R)          # (N,3 rows of d, 3 components)
        return np.transpose(sol, (0, 2, 1))  # Tensor3 rows = component gradients
    np.add.at(R, ob, wgt[:, None] * d * diff[:, None])
    return np.linalg.solve(M, R[:, :, None])[:, :, 0]


def gradient(field: Field, method: str):
    if method == "greenGauss":
        return gradient_green_gauss(field)
    if method == "leastSquares":
        return gradient_least_squares(field)
    raise ValueError(method)


def interpolate(field: Field, method: str, grad_method: str, outward_flux=None):
    """interpolate (operators.cpp:705-745)."""
    if method == "linear":
        return interpolate_linear(field, outward_flux)
    return corrected_face_values(field, gradient(field, grad_method), outward_flux)


class LDU:
    """DiscreteEquation<T> storage (include/babelsim/discrete_equation.h:14-50)."""

    def __init__(self, geo, vector):
        self.geo = geo
        self.vector = vector
        self.diag = np.zeros(geo.n_cells)
        self.upper = np.zeros(geo.n_faces)
        self.lower = np.zeros(geo.n_faces)
        self.source = np.zeros((geo.n_cells, 3)) if vector else np.zeros(geo.n_cells)

    def copy(self):
        c = LDU(self.geo, self.vector)
        c.diag, c.upper, c.lower, c.source = self.diag.copy(), self.upper.copy(), self.lower.copy(), self.source.copy()
        return c

    def accumulate(self, other, f):
        """accumulate (procedural_equation.cpp:62-70)."""
        self.diag += f * other.diag
        self.source += f * other.source
        self.upper += f * other.upper
        self.lower += f * other.lower

    def apply(self, x):
        """equ::apply LDU product (procedural_equation.cpp:281-292)."""
        geo = self.geo
        y = (self.diag[:, None] * x) if x.ndim == 2 else self.diag * x
        inn = np.nonzero(geo.neighbour >= 0)[0]
        o, n = geo.owner[inn], geo.neighbour[inn]
        if x.ndim == 2:
            np.add.at(y, o, self.upper[inn][:, None] * x[n])
            np.add.at(y, n, self.lower[inn][:, None] * x[o])
        else:
            np.add.at(y, o, self.upper[inn] * x[n])
            np.add.at(y, n, self.lower[inn] * x[o])
        return y

    def matrix(self):
        """Sparse matrix of the LDU system (row = cell)."""
        import scipy.sparse as sp
        geo = self.geo
        inn = np.nonzero(geo.neighbour >= 0)[0]
        o, n = geo.owner[inn], geo.neighbour[inn]
        rows = np.concatenate([np.arange(geo.n_cells), o, n])
        cols = np.concatenate([np.arange(geo.n_cells), n, o])
        vals = np.concatenate([self.diag, self.upper[inn], self.lower[inn]])
        return sp.csr_matrix((vals, (rows, cols)), shape=(geo.n_cells, geo.n_cells))


def add_convection(eq: LDU, phi, x: Field, method, interp_method, grad_method, scale=1.0):
    """addConvectionImpl (operators.cpp:535-661)."""
    geo = eq.geo
    x.flux = np.array(phi, dtype=np.float64)  # setBoundaryFlux
    g = None
    if method == "linearUpwind" or (method == "central" and interp_method == "corrected"):
        g = gradient(x, grad_method)
    F = scale * phi
    inn = np.nonzero(geo.neighbour >= 0)[0]
    o, n = geo.owner[inn], geo.neighbour[inn]
    Fi = F[inn]
    vec = x.vector

    def addsrc(cells, val):
        np.add.at(eq.source, cells, val)
    if method in ("upwind", "linearUpwind"):
        np.add.at(eq.diag, o, np.maximum(Fi, 0.0))
        eq.upper[inn] += np.minimum(Fi, 0.0)
        np.add.at(eq.diag, n, np.maximum(-Fi, 0.0))
        eq.lower[inn] += np.minimum(-Fi, 0.0)
        if method == "linearUpwind":
            up = np.where(Fi >= 0.0, o, n)
            off = geo.xf[inn] - geo.xc[up]
            corr = np.einsum("fcj,fj->fc", g[up], off) if vec else np.einsum("fj,fj->f", g[up], off)
            fc = Fi[:, None] * corr if vec else Fi * corr
            addsrc(o, -fc)
            addsrc(n, fc)
    elif method == "central":
        w = geo.weight[inn]
        np.add.at(eq.diag, o, Fi * w)
        eq.upper[inn] += Fi * (1.0 - w)
        eq.lower[inn] -= Fi * w
        np.add.at(eq.diag, n, -(Fi * (1.0 - w)))
        if g is not None:
            corr = corrected_interior(x, g, inn) - (
                w[:, None] * x.v[o] + (1.0 - w)[:, None] * x.v[n] if vec else w * x.v[o] + (1.0 - w) * x.v[n])
            fc = Fi[:, None] * corr if vec else Fi * corr
            addsrc(o, -fc)
            addsrc(n, fc)
    else:
        raise ValueError(method)
    bf = _bfaces(geo)
    ob = geo.owner[bf]
    Fb = F[bf]
    types, values = face_condition(x, bf, Fb)
    if method in ("upwind", "linearUpwind"):
        pos = Fb >= 0.0
        np.add.at(eq.diag, ob[pos], Fb[pos])
        if method == "linearUpwind":
            off = geo.xf[bf][pos] - geo.xc[ob[pos]]
            gg = g[ob[pos]]
            corr = np.einsum("fcj,fj->fc", gg, off) if vec else np.einsum("fj,fj->f", gg, off)
            addsrc(ob[pos], -(Fb[pos][:, None] * corr if vec else Fb[pos] * corr))
        neg = ~pos
        bv = boundary_trace(x, bf[neg], Fb[neg])
        addsrc(ob[neg], -(Fb[neg][:, None] * bv if vec else Fb[neg] * bv))
        return
    # central
    for t in (FIXED_VALUE, FIXED_GRADIENT, ZERO_GRADIENT, SYMMETRY):
        m = types == t
        if not np.any(m):
            continue
        if t == FIXED_VALUE:
            addsrc(ob[m], -(Fb[m][:, None] * values[m] if vec else Fb[m] * values[m]))
        elif t == FIXED_GRADIENT:
            dist = _boundary_normal_distance(geo, bf[m])
            np.add.at(eq.diag, ob[m], Fb[m])
            addsrc(ob[m], -((Fb[m] * dist)[:, None] * values[m] if vec else Fb[m] * dist * values[m]))
        else:
            np.add.at(eq.diag, ob[m], Fb[m])
    if g is not None:
        corr = reconstructed_boundary(x, g, bf, Fb) - boundary_trace(x, bf, Fb)
        addsrc(ob, -(Fb[:, None] * corr if vec else Fb * corr))


def _limit(orth, corr, method):
    """limitNonOrthogonalCorrection (operators.cpp:499-513)."""
    if method == "corrected":
        return corr
    if method == "limitedCorrected":
        b = np.abs(orth)
        return np.clip(corr, -b, b)
    return np.zeros_like(corr)


def integrated_normal_gradient(x: Field, g, method):
    """integratedNormalGradient scalar (operators.cpp:857-902) over all faces."""
    geo = x.geo
    out = np.zeros(geo.n_faces)
    inn = np.nonzero(geo.neighbour >= 0)[0]
    o, n = geo.owner[inn], geo.neighbour[inn]
    orth = geo.dcoef[inn] * (x.v[n] - x.v[o])
    out[inn] = orth
    corrected = method in ("corrected", "limitedCorrected")
    if corrected:
        fg = _face_grad(geo, g, inn)
        out[inn] = orth + _limit(orth, np.einsum("ij,ij->i", geo.kvec[inn], fg), method)
    bf = _bfaces(geo)
    types, values = face_condition(x, bf)
    fgm = types == FIXED_GRADIENT
    out[bf[fgm]] = values[fgm] * geo.area[bf[fgm]]
    fv = types == FIXED_VALUE
    f = bf[fv]
    ob = geo.owner[f]
    orth = geo.dcoef[f] * (values[fv] - x.v[ob])
    out[f] = orth
    if corrected:
        out[f] = orth + _limit(orth, np.einsum("ij,ij->i", geo.kvec[f], g[ob]), method)
    return out


def integrated_normal_gradient_vector(x: Field, g, method):
    """integratedNormalGradient vector (operators.cpp:904-954) over all faces."""
    geo = x.geo
    out = np.zeros((geo.n_faces, 3))
    inn = np.nonzero(geo.neighbour >= 0)[0]
    o, n = geo.owner[inn], geo.neighbour[inn]
    orth = geo.dcoef[inn][:, None] * (x.v[n] - x.v[o])
    out[inn] = orth
    corrected = method in ("corrected", "limitedCorrected")
    if corrected:
        fg = _face_grad(geo, g, inn)
        corr = np.einsum("fcj,fj->fc", fg, geo.kvec[inn])
        out[inn] = orth + _limit(orth, corr, method)
    bf = _bfaces(geo)
    types, values = face_condition(x, bf)
    fgm = types == FIXED_GRADIENT
    out[bf[fgm]] = geo.area[bf[fgm]][:, None] * values[fgm]
    m = (types == FIXED_VALUE) | (types == SYMMETRY)
    f = bf[m]
    ob = geo.owner[f]
    bv = boundary_trace(x, f)
    orth = geo.dcoef[f][:, None] * (bv - x.v[ob])
    out[f] = orth
    if corrected:
        nrm = geo.normal[f]
        sym = (types[m] == SYMMETRY)
        for c in range(3):
            gb = g[ob][:, c, :].copy()
            gb[sym] -= np.einsum("ij,ij->i", gb[sym], nrm[sym])[:, None] * nrm[sym]
            out[f, c] = orth[:, c] + _limit(orth[:, c], np.einsum("ij,ij->i", geo.kvec[f], gb), method)
    return out


def add_diffusion(eq: LDU, gamma_f, x: Field, g, method):
    """addScalarDiffusion / addVectorDiffusion (operators.cpp:1287-1438); g is the frozen gradient."""
    geo = eq.geo
    if np.any(gamma_f < 0.0) or not np.all(np.isfinite(gamma_f)):
        raise ValueError("face diffusivity must be non-negative and finite")
    corrected = method in ("corrected", "limitedCorrected")
    vec = x.vector
    inn = np.nonzero((geo.neighbour >= 0) & (gamma_f != 0.0))[0]
    o, n = geo.owner[inn], geo.neighbour[inn]
    gam = gamma_f[inn]
    c = gam * geo.dcoef[inn]
    np.add.at(eq.diag, o, c)
    np.add.at(eq.diag, n, c)
    eq.upper[inn] -= c
    eq.lower[inn] -= c
    if corrected:
        if vec:
            ing = integrated_normal_gradient_vector(x, g, method)[inn]
            orth = geo.dcoef[inn][:, None] * (x.v[n] - x.v[o])
            corr = gam[:, None] * (ing - orth)
        else:
            ing = integrated_normal_gradient(x, g, method)[inn]
            orth = geo.dcoef[inn] * (x.v[n] - x.v[o])
            corr = gam * (ing - orth)
        np.add.at(eq.source, o, corr)
        np.add.at(eq.source, n, -corr)
    bf = np.nonzero((geo.neighbour < 0) & (gamma_f != 0.0))[0]
    types, values = face_condition(x, bf)
    ob = geo.owner[bf]
    gam = gamma_f[bf]
    c = gam * geo.dcoef[bf]
    if vec:
        m = (types == FIXED_VALUE) | (types == SYMMETRY)
        bv = boundary_trace(x, bf[m], -1.0)
        np.add.at(eq.diag, ob[m], c[m])
        np.add.at(eq.source, ob[m], c[m][:, None] * bv)
        if corrected:
            ing = integrated_normal_gradient_vector(x, g, method)[bf[m]]
            orth = geo.dcoef[bf[m]][:, None] * (bv - x.v[ob[m]])
            np.add.at(eq.source, ob[m], gam[m][:, None] * (ing - orth))
        fg = types == FIXED_GRADIENT
        np.add.at(eq.source, ob[fg], (gam[fg] * geo.area[bf[fg]])[:, None] * values[fg])
    else:
        m = types == FIXED_VALUE
        np.add.at(eq.diag, ob[m], c[m])
        np.add.at(eq.source, ob[m], c[m] * values[m])
        if corrected:
            ing = integrated_normal_gradient(x, g, method)[bf[m]]
            orth = geo.dcoef[bf[m]] * (values[m] - x.v[ob[m]])
            np.add.at(eq.source, ob[m], gam[m] * (ing - orth))
        fg = types == FIXED_GRADIENT
        np.add.at(eq.source, ob[fg], gam[fg] * values[fg] * geo.area[bf[fg]])


def diffusion_flux(gamma_f, x: Field, g, method):
    """diffusionFlux (operators.cpp:1004-1024)."""
    return gamma_f * integrated_normal_gradient(x, g, method)


class Equation:
    """equ::Equation<T> state (procedural_equation.cpp:15-34)."""

    def __init__(self, x: Field, options: dict, term_options: dict):
        self.x = x
        self.options = options              # base options for the equation
        self.term_options = term_options    # term -> options (already overlaid)
        self.ldu = LDU(x.geo, x.vector)
        self.diffusion = []                 # list of (kf, boundary field, correction, factor)
        self.boundary_flux = None

    def opts(self, term=None):
        return self.term_options.get(term, self.options) if term else self.options

    def reset(self):
        self.ldu = LDU(self.x.geo, self.x.vector)
        self.diffusion = []
        self.boundary_flux = None


def eq_div(eq: Equation, phi, factor=1.0, term=None):
    """equ::div (procedural_equation.cpp:116-129)."""
    m = eq.opts(term)
    eq.boundary_flux = phi
    add_convection(eq.ldu, phi, eq.x, m["convection"], m["interpolation"], m["gradient"], factor)


def eq_laplacian(eq: Equation, k, factor, term=None):
    """equ::laplacian with a cell or face coefficient (procedural_equation.cpp:130-176).

    ``k`` is a Field (cell coefficient, interpolated with the coefficient
    options), an array of face values (used as given) or a float (constant).
    """
    m = eq.opts(term)
    x = eq.x
    geo = x.geo
    if isinstance(k, Field):
        kf = interpolate(k, m.get("coefficientInterpolation") or m["interpolation"],
                         m.get("coefficientGradient") or m["gradient"])
    elif isinstance(k, np.ndarray):
        kf = np.array(k, dtype=np.float64)   # a face coefficient is used as given
    else:
        kf = np.full(geo.n_faces, float(k))
    contrib = LDU(geo, x.vector)
    g = None
    if m["diffusion"] != "orthogonal":
        g = gradient(x, m["gradient"])
    add_diffusion(contrib, kf, x, g, m["diffusion"])
    if not x.vector:
        if m["diffusion"] == "orthogonal":
            corr = np.zeros(geo.n_faces)
        else:
            corr = diffusion_flux(kf, x, g, m["diffusion"]) - diffusion_flux(kf, x, g, "orthogonal")
        eq.diffusion.append((kf, x.copy(), corr, factor))
    eq.ldu.accumulate(contrib, -factor)


def eq_source(eq: Equation, values, factor=1.0):
    """equ::source with a cell field (procedural_equation.cpp:192-196): b += factor V value."""
    geo = eq.x.geo
    if eq.x.vector:
        eq.ldu.source += factor * geo.volume[:, None] * values
    else:
        eq.ldu.source += factor * geo.volume * values


def eq_relax(eq: Equation, previous, alpha):
    """equ::relax (procedural_equation.cpp:298-305)."""
    q = eq.ldu
    extra = q.diag * (1.0 / alpha - 1.0)
    q.diag = q.diag + extra
    q.source = q.source + (extra[:, None] * previous if previous.ndim == 2 else extra * previous)


def eq_scale(eq: Equation, f):
    """equ::scale (procedural_equation.cpp:240-247)."""
    q = eq.ldu
    q.diag = q.diag * f
    q.upper = q.upper * f
    q.lower = q.lower * f
    q.source = f * q.source
    eq.diffusion = [(kf, b, c, fac * f) for (kf, b, c, fac) in eq.diffusion]


def eq_reference_if_unanchored(eq: Equation, value=0.0):
    """equ::reference(Equation, value) (procedural_equation.cpp:316-333, 306-315)."""
    q = eq.ldu
    geo = eq.x.geo
    row = q.diag.copy()
    mag = np.abs(q.diag)
    inn = np.nonzero(geo.neighbour >= 0)[0]
    o, n = geo.owner[inn], geo.neighbour[inn]
    np.add.at(row, o, q.upper[inn])
    np.add.at(mag, o, np.abs(q.upper[inn]))
    np.add.at(row, n, q.lower[inn])
    np.add.at(mag, n, np.abs(q.lower[inn]))
    constant = np.all(np.isfinite(row) & (np.abs(row) <= 64 * EPS * mag))
    if constant:
        if not q.diag[0] > 0:
            raise ValueError("reference requires a positive diagonal")
        q.source[0] += q.diag[0] * value
        q.diag[0] *= 2
    return bool(constant)


def eq_face_flux(eq: Equation, solution_values):
    """equ::faceFlux (procedural_equation.cpp:335-352)."""
    geo = eq.x.geo
    out = np.zeros(geo.n_faces)
    for kf, boundary, corr, factor in eq.diffusion:
        val = boundary.with_values(solution_values)
        inc = diffusion_flux(kf, val, None, "orthogonal") + corr
        out += factor * inc
    return out


def relative_residual(ldu: LDU, x):
    """diagnostics::relativeResidual (procedural_equation.cpp:429-433)."""
    ax = ldu.apply(x)
    r = ldu.source - ax
    nr, na, nb = (np.sqrt(np.sum(v * v)) for v in (r, ax, ldu.source))
    return nr / max(na + nb, 1e-30)


def flux(U: Field, interp_method, grad_method):
    """flux of a cell vector (operators.cpp:957-1002), saving the new boundary-flux context."""
    geo = U.geo
    if U.flux is None:
        bf = _bfaces(geo)
        init = np.zeros(geo.n_faces)
        init[bf] = np.einsum("ij,ij->i", U.v[geo.owner[bf]], geo.Sf[bf])
        U.flux = init
    if interp_method == "corrected":
        fv = corrected_face_values(U, gradient(U, grad_method))
    else:
        fv = interpolate_linear(U)
    out = np.einsum("ij,ij->i", fv, geo.Sf)
    U.flux = out.copy()   # FvmExecution::evaluate(FaceFlux) (fvm_execution.cpp:269-280)
    return out


def divergence_flux(geo, phi):
    """divergence of an integrated face flux (operators.cpp:1055-1063)."""
    out = np.zeros(geo.n_cells)
    inn = geo.neighbour >= 0
    np.add.at(out, geo.owner, phi / geo.volume[geo.owner])
    np.add.at(out, geo.neighbour[inn], -phi[inn] / geo.volume[geo.neighbour[inn]])
    return out


def normal_gradient(x: Field, g, method):
    """NormalGradient (fvm_execution.cpp:522-543): integratedNormalGradient / |Sf|."""
    return integrated_normal_gradient(x, g, method) / x.geo.area


def flux_balance(geo, phi):
    """fluxBalance (fvm_execution.cpp:149-177): returns dict(l1, l2, maximum, relative)."""
    imb = np.zeros(geo.n_cells)
    scale = np.zeros(geo.n_cells)
    inn = geo.neighbour >= 0
    np.add.at(imb, geo.owner, phi)
    np.add.at(imb, geo.neighbour[inn], -phi[inn])
    np.add.at(scale, geo.owner, np.abs(phi))
    np.add.at(scale, geo.neighbour[inn], np.abs(phi[inn]))
    l1 = float(np.sum(np.abs(imb)))
    return dict(l1=l1, l2=float(np.sqrt(np.sum(imb * imb))), maximum=float(np.max(np.abs(imb))),
                relative=l1 / max(float(np.sum(scale)), 1e-30))


def relative_change(cur, prev):
    """relativeChange (fvm_execution.cpp:91-128)."""
    return float(np.sqrt(np.sum((cur - prev) ** 2)) / max(np.sqrt(np.sum(cur * cur)), 1e-30))


def relative_magnitude(v, ref):
    """relativeMagnitude (fvm_execution.cpp:130-147)."""
    return float(np.sqrt(np.sum(v * v)) / max(np.sqrt(np.sum(ref * ref)), 1e-30))


def homogeneous_bcs(bcs):
    """setHomogeneousCorrectionBoundaries (field.h:380-405)."""
    out = []
    for t, _ in bcs:
        if t == FIXED_VALUE:
            out.append((FIXED_VALUE, 0.0))
        elif t == SYMMETRY:
            out.append((SYMMETRY, 0.0))
        else:
            out.append((ZERO_GRADIENT, 0.0))
    return out
