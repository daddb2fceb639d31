"""Python host API over the C ABI: contexts, meshes, fields, equations, SIMPLE.

Mirrors the reference's SDK vocabulary (Field, equ::/math:: operators,
LinearSolverConfig, SolveResult) one call per C entry point.  Every call goes
through libbabelsim_b200.so; there is no other implementation.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (KEpsilonConfig, KOmegaConfig, PisoTurbulenceControls, SaConfig, MeshGeometry, Options, PisoConfig, PisoReport, SimpleConfig, SimpleReport, SolveResult, SolverConfig,
                   SystemCounters, check, f64, i32, lib, ptr)

BC = {"fixedValue": 0, "fixedGradient": 1, "zeroGradient": 2, "inletOutlet": 3, "symmetry": 4}
INTERP = {"linear": 0, "corrected": 1}
GRAD = {"greenGauss": 0, "leastSquares": 1}
CONV = {"upwind": 0, "linearUpwind": 1, "central": 2}
DIFF = {"orthogonal": 0, "corrected": 1, "limitedCorrected": 2}
KSP = {"cg": 0, "bcgs": 1, "gmres": 2, "fgmres": 3}
PC = {"none": 0, "icc": 1, "hypre": 2, "gamg": 3, "bjacobi": 4, "asm": 5, "jacobi": 6}


def options(interpolation="linear", gradient="greenGauss", convection="upwind", diffusion="orthogonal",
            coefficient_interpolation=None, coefficient_gradient=None) -> Options:
    return Options(INTERP[interpolation], GRAD[gradient], CONV[convection], DIFF[diffusion],
                   -1 if coefficient_interpolation is None else INTERP[coefficient_interpolation],
                   -1 if coefficient_gradient is None else GRAD[coefficient_gradient])


def locality_order(poly):
    """(order, applied): the cell numbering the library uses inside for this polyhedral mesh,
    order[internal] = caller cell (reverse Cuthill-McKee when the caller's order is poor)."""
    owner, nbr = i32(poly.owner), i32(poly.neighbour)
    n = poly.n_cells
    order = np.zeros(n, np.int32)
    applied = C.c_int32()
    check(lib().bsg_mesh_locality_order(n, len(owner), ptr(owner), ptr(nbr), ptr(order), C.byref(applied)))
    return order, bool(applied.value)


def file_info(path) -> dict:
    """Host-only read of a BABELSIM_MESH 3 file by the native reader: sizes and patches."""
    out = np.zeros(4, np.int64)
    buf = C.create_string_buffer(1 << 20)
    check(lib().bsg_mesh_file_info(str(path).encode(), ptr(out), buf, len(buf)))
    lines = [ln.split() for ln in buf.value.decode().splitlines() if ln.strip()]
    return {"cells": int(out[0]), "faces": int(out[1]), "vertices": int(out[2]),
            "patches": [(ln[0], ln[1]) for ln in lines]}


def solver_config(ksp="cg", pc="jacobi", atol=1e-14, rtol=1e-10, max_iterations=1000, warm_start=False,
                  amg_max_levels=12, amg_coarse_size=400, amg_smoothing_steps=1, precision=0, rebuild_interval=8,
                  reuse_growth=2.0) -> SolverConfig:
    return SolverConfig(KSP[ksp], PC[pc], atol, rtol, max_iterations, int(warm_start), rebuild_interval, reuse_growth,
                        amg_max_levels, amg_coarse_size, amg_smoothing_steps, precision)


class Context:
    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().bsg_context_create(device, C.byref(h)))
        self.h = h

    def launches(self) -> int:
        v = C.c_int64()
        check(lib().bsg_context_launches(self.h, C.byref(v)), self.h)
        return v.value

    def synchronize(self):
        check(lib().bsg_context_synchronize(self.h), self.h)

    def profile(self, enable: bool):
        check(lib().bsg_context_profile(self.h, int(enable)), self.h)

    def profile_report(self) -> dict:
        import json
        buf = C.create_string_buffer(1 << 16)
        check(lib().bsg_context_profile_report(self.h, buf, len(buf)), self.h)
        # name -> (launches, total ms, algorithmic bytes, work units such as Krylov iterations)
        return {k: (int(v[0]), float(v[1]), float(v[2]), float(v[3])) for k, v in json.loads(buf.value.decode()).items()}

    def phase_log(self, capacity: int):
        """Enable (capacity > 0) or disable the persistent-kernel phase timeline."""
        check(lib().bsg_context_phase_log(self.h, capacity), self.h)

    def phase_log_read(self, capacity: int = 1 << 20):
        """[(phase id, ns)] recorded since the last read (device globaltimer)."""
        buf = np.zeros(2 * capacity, np.int64)
        n = C.c_int32()
        check(lib().bsg_context_phase_log_read(self.h, ptr(buf), capacity, C.byref(n)), self.h)
        return buf[:2 * n.value].reshape(-1, 2)

    def record(self, slot: int):
        check(lib().bsg_context_event_record(self.h, slot), self.h)

    def elapsed_ms(self, a: int, b: int) -> float:
        v = C.c_double()
        check(lib().bsg_context_event_elapsed(self.h, a, b, C.byref(v)), self.h)
        return v.value

    def close(self):
        if self.h:
            lib().bsg_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def validate_polyhedral(poly):
    """Run the library's host geometry on a polyhedral mesh (no device); returns (n_cells, orthogonal)."""
    off, ids = poly.flat() if hasattr(poly, "flat") else (
        np.concatenate([[0], np.cumsum([len(f) for f in poly.faces])]), np.concatenate(poly.faces))
    verts, off, ids = f64(poly.vertices), i32(off), i32(ids)
    owner, nbr, patch = i32(poly.owner), i32(poly.neighbour), i32(poly.patch)
    nc, orth = C.c_int32(), C.c_int32()
    check(lib().bsg_mesh_validate_polyhedral(len(verts), ptr(verts), len(owner), ptr(off), ptr(ids), ptr(owner),
                                             ptr(nbr), ptr(patch), len(poly.patch_names), C.byref(nc),
                                             C.byref(orth)))
    return nc.value, bool(orth.value)


class Mesh:
    """A device-resident mesh (bsg_mesh)."""

    def __init__(self, ctx: Context, handle, n_patches):
        self.ctx = ctx
        self.h = handle
        sizes = np.zeros(5, np.int64)
        check(lib().bsg_mesh_sizes(self.h, ptr(sizes)), ctx.h)
        self.n_cells, self.n_faces, self.n_interior, self.n_patches, orth = (int(v) for v in sizes)
        self.orthogonal = bool(orth)

    @classmethod
    def from_polyhedral(cls, ctx: Context, poly, host_geometry: bool = False):
        """Geometry computed by the library from a polyhedral description (see meshgen.PolyMesh),
        on the device (default) or on the host (`host_geometry`); both give identical bits."""
        off, ids = poly.flat() if hasattr(poly, "flat") else (
            np.concatenate([[0], np.cumsum([len(f) for f in poly.faces])]), np.concatenate(poly.faces))
        offsets, ids = i32(off), i32(ids)
        verts = f64(poly.vertices)
        owner, nbr, patch = i32(poly.owner), i32(poly.neighbour), i32(poly.patch)
        h = C.c_void_p()
        create = lib().bsg_mesh_create_polyhedral_host if host_geometry else lib().bsg_mesh_create_polyhedral
        check(create(ctx.h, len(verts), ptr(verts), len(owner), ptr(offsets), ptr(ids), ptr(owner), ptr(nbr),
                     ptr(patch), len(poly.patch_names), C.byref(h)), ctx.h)
        m = cls(ctx, h, len(poly.patch_names))
        m.patch_names = list(poly.patch_names)
        return m

    @classmethod
    def from_file(cls, ctx: Context, path: str):
        """The reference's mesh file (BABELSIM_MESH 3) read by the library's native reader,
        geometry on the device."""
        info = file_info(path)
        h = C.c_void_p()
        check(lib().bsg_mesh_create_from_file(ctx.h, str(path).encode(), C.byref(h)), ctx.h)
        m = cls(ctx, h, len(info["patches"]))
        m.patch_names = [name for name, _ in info["patches"]]
        return m

    @classmethod
    def from_geometry(cls, ctx: Context, geo: dict, n_patches: int):
        """Geometry supplied by the caller (the reference's MeshStorage arrays)."""
        keep = {k: (i32(v) if k in ("face_owner", "face_neighbour", "face_patch") else f64(v)) for k, v in geo.items()
                if k != "orthogonal_geometry"}
        g = MeshGeometry(len(keep["cell_volumes"]), len(keep["face_owner"]), n_patches,
                         *(ptr(keep[k]) for k in ("face_owner", "face_neighbour", "face_patch", "face_area_vectors",
                                                  "face_centres", "face_areas", "face_normals", "face_owner_weights",
                                                  "face_orthogonal_coefficients", "face_non_orthogonal",
                                                  "face_skewness", "cell_centres", "cell_volumes")),
                         int(np.asarray(geo["orthogonal_geometry"]).ravel()[0]))
        h = C.c_void_p()
        check(lib().bsg_mesh_create(ctx.h, C.byref(g), C.byref(h)), ctx.h)
        return cls(ctx, h, n_patches)

    def export(self, name: str) -> np.ndarray:
        width = {"face_owner": 1, "face_neighbour": 1, "face_patch": 1, "face_areas": 1, "face_owner_weights": 1,
                 "face_orthogonal_coefficients": 1, "cell_volumes": 1}.get(name, 3)
        count = self.n_cells if name.startswith("cell_") else self.n_faces
        dtype = np.int32 if name in ("face_owner", "face_neighbour", "face_patch") else np.float64
        out = np.zeros(count * width, dtype)
        check(lib().bsg_mesh_export(self.h, name.encode(), ptr(out)), self.ctx.h)
        return out.reshape(count, width) if width == 3 else out

    def close(self):
        if self.h:
            lib().bsg_mesh_destroy(self.h)
            self.h = None


class Field:
    """Device field (bsg_field): location 'cell' or 'face', 1/3/9 components."""

    def __init__(self, mesh: Mesh, location="cell", components=1, values=None):
        self.mesh = mesh
        self.location = location
        self.components = components
        h = C.c_void_p()
        check(lib().bsg_field_create(mesh.h, 0 if location == "cell" else 1, components, C.byref(h)), mesh.ctx.h)
        self.h = h
        if values is not None:
            self.upload(values)

    @property
    def count(self):
        return self.mesh.n_cells if self.location == "cell" else self.mesh.n_faces

    def set_boundary(self, patch: int, kind: str, value=0.0):
        v = f64(np.broadcast_to(np.asarray(value, dtype=np.float64), (3,)) if np.ndim(value) == 0 else
                np.pad(np.asarray(value, np.float64), (0, 3 - len(value))))
        check(lib().bsg_field_set_boundary(self.h, patch, BC[kind], ptr(v)), self.mesh.ctx.h)

    def upload(self, values):
        v = f64(values).reshape(-1)
        assert v.size == self.count * self.components
        check(lib().bsg_field_upload(self.h, ptr(v)), self.mesh.ctx.h)

    def download(self) -> np.ndarray:
        out = np.zeros(self.count * self.components)
        check(lib().bsg_field_download(self.h, ptr(out)), self.mesh.ctx.h)
        return out if self.components == 1 else out.reshape(self.count, self.components)

    def set_boundary_flux(self, face_flux: "Field"):
        check(lib().bsg_field_set_boundary_flux(self.h, face_flux.h), self.mesh.ctx.h)

    def close(self):
        if self.h:
            lib().bsg_field_destroy(self.h)
            self.h = None


def grad(x: Field, method="greenGauss") -> Field:
    out = Field(x.mesh, "cell", 3 * x.components)
    check(lib().bsg_math_grad(x.h, GRAD[method], out.h), x.mesh.ctx.h)
    return out


def interpolate(x: Field, opts: Options) -> Field:
    out = Field(x.mesh, "face", x.components)
    check(lib().bsg_math_interpolate(x.h, C.byref(opts), out.h), x.mesh.ctx.h)
    return out


def flux(U: Field, opts: Options) -> Field:
    out = Field(U.mesh, "face", 1)
    check(lib().bsg_math_flux(U.h, C.byref(opts), out.h), U.mesh.ctx.h)
    return out


def div_flux(phi: Field) -> Field:
    out = Field(phi.mesh, "cell", 1)
    check(lib().bsg_math_div_flux(phi.h, out.h), phi.mesh.ctx.h)
    return out


def normal_gradient(x: Field, opts: Options, gradient: Field | None = None) -> Field:
    out = Field(x.mesh, "face", 1)
    check(lib().bsg_math_normal_gradient(x.h, gradient.h if gradient else None, C.byref(opts), out.h), x.mesh.ctx.h)
    return out


class Equation:
    """equ::Equation on the device (bsg_equation)."""

    def __init__(self, unknown: Field, opts: Options):
        self.x = unknown
        h = C.c_void_p()
        check(lib().bsg_equation_create(unknown.h, C.byref(opts), C.byref(h)), unknown.mesh.ctx.h)
        self.h = h

    def _c(self, code):
        check(code, self.x.mesh.ctx.h)

    def reset(self):
        self._c(lib().bsg_equ_reset(self.h))

    def div(self, phi: Field, scale=1.0, term: Options | None = None):
        self._c(lib().bsg_equ_div(self.h, phi.h, scale, C.byref(term) if term else None))

    def laplacian(self, coefficient, factor, term: Options | None = None):
        if isinstance(coefficient, Field):
            self._c(lib().bsg_equ_laplacian(self.h, coefficient.h, 0.0, factor, C.byref(term) if term else None))
        else:
            self._c(lib().bsg_equ_laplacian(self.h, None, float(coefficient), factor, C.byref(term) if term else None))

    def source(self, value: Field, factor=1.0):
        self._c(lib().bsg_equ_source(self.h, value.h, factor))

    def ddt(self, capacity, previous: Field, dt: float, method="euler", older: Field | None = None,
            older_dt: float = 0.0):
        """equ::ddt with explicit levels; capacity is a cell Field or a number."""
        m = {"steady": 0, "euler": 1, "bdf2": 2}[method.lower()]
        cap = capacity.h if isinstance(capacity, Field) else None
        c = 0.0 if isinstance(capacity, Field) else float(capacity)
        self._c(lib().bsg_equ_ddt(self.h, cap, c, previous.h, older.h if older else None, dt, older_dt, m))

    def reaction(self, coefficient, factor=1.0):
        """equ::reaction: diagonal += factor*coefficient*V (coefficient: cell Field or number)."""
        if isinstance(coefficient, Field):
            self._c(lib().bsg_equ_reaction(self.h, coefficient.h, 0.0, factor))
        else:
            self._c(lib().bsg_equ_reaction(self.h, None, float(coefficient), 1.0))

    def apply(self, x: Field) -> Field:
        out = Field(self.x.mesh, "cell", self.x.components)
        self._c(lib().bsg_equ_apply(self.h, x.h, out.h))
        return out

    def residual(self, x: Field) -> Field:
        out = Field(self.x.mesh, "cell", self.x.components)
        self._c(lib().bsg_equ_residual(self.h, x.h, out.h))
        return out

    def relax(self, previous: Field, alpha):
        self._c(lib().bsg_equ_relax(self.h, previous.h, alpha))

    def scale(self, f):
        self._c(lib().bsg_equ_scale(self.h, f))

    def reference_if_unanchored(self, value=0.0) -> bool:
        flag = C.c_int32()
        self._c(lib().bsg_equ_reference_if_unanchored(self.h, value, C.byref(flag)))
        return bool(flag.value)

    def face_flux(self, solution: Field) -> Field:
        out = Field(self.x.mesh, "face", 1)
        self._c(lib().bsg_equ_face_flux(self.h, solution.h, out.h))
        return out

    def relative_residual(self, x: Field) -> float:
        v = C.c_double()
        self._c(lib().bsg_equ_relative_residual(self.h, x.h, C.byref(v)))
        return v.value

    def solve(self, cfg: SolverConfig):
        res = (SolveResult * self.x.components)()
        self._c(lib().bsg_equ_solve(self.h, C.byref(cfg), res))
        return list(res)

    def download(self):
        m = self.x.mesh
        d, u, l = np.zeros(m.n_cells), np.zeros(m.n_faces), np.zeros(m.n_faces)
        s = np.zeros(m.n_cells * self.x.components)
        self._c(lib().bsg_equ_download(self.h, ptr(d), ptr(u), ptr(l), ptr(s)))
        return dict(diag=d, upper=u, lower=l, source=s if self.x.components == 1 else s.reshape(-1, 3))

    def close(self):
        if self.h:
            lib().bsg_equation_destroy(self.h)
            self.h = None


def solve_ldu(mesh: Mesh, cfg: SolverConfig, diag, upper, lower, source, x0=None):
    """ComputeBackend::solve on host LDU arrays (bsg_solve_ldu)."""
    src = f64(source)
    comps = 1 if src.ndim == 1 else 3
    x = f64(np.zeros_like(src) if x0 is None else x0).copy()
    res = (SolveResult * comps)()
    check(lib().bsg_solve_ldu(mesh.h, C.byref(cfg), comps, ptr(f64(diag)), ptr(f64(upper)), ptr(f64(lower)),
                              ptr(src), ptr(x), res), mesh.ctx.h)
    return x, list(res)


class LinearSystem:
    """One equation's persistent linear system (bsg_system; PetscLinearSystem's lifecycle):
    buffers and the AMG structure made once, exactly unchanged matrices skipped, AMG
    hierarchies lagged and rebuilt on the reference's schedule."""

    def __init__(self, mesh: Mesh, components: int = 1):
        self.mesh, self.components = mesh, components
        h = C.c_void_p()
        check(lib().bsg_system_create(mesh.h, components, C.byref(h)), mesh.ctx.h)
        self.h = h

    def solve(self, cfg: SolverConfig, diag, upper, lower, source, x0=None):
        src = f64(source)
        x = f64(np.zeros_like(src) if x0 is None else x0).copy()
        res = (SolveResult * self.components)()
        check(lib().bsg_system_solve(self.h, C.byref(cfg), ptr(f64(diag)), ptr(f64(upper)), ptr(f64(lower)),
                                     ptr(src), ptr(x), res), self.mesh.ctx.h)
        return x, list(res)

    def counters(self) -> dict:
        k = SystemCounters()
        check(lib().bsg_system_counters_read(self.h, C.byref(k)), self.mesh.ctx.h)
        return {name: getattr(k, name) for name, _ in k._fields_}

    def close(self):
        if self.h:
            lib().bsg_system_destroy(self.h)
            self.h = None


class _TurbulenceModels:
    """rans::load for a flow solver (src/physics/RANS/model.cpp:24-53): k-omega, k-epsilon or
    Spalart-Allmaras, its boundary conditions, initial fields and outputs.  Subclasses name their C
    entry-point prefix."""
    _prefix = ""

    def _fn(self, name):
        return getattr(lib(), self._prefix + name)

    def _enable(self, model, cfg):
        check(self._fn("enable_" + model)(self.h, C.byref(cfg)), self.mesh.ctx.h)

    def enable_komega(self, beta_star=0.09, beta=0.075, gamma=5.0 / 9.0, sigma_k=0.5, sigma_omega=0.5, k_min=1e-12,
                      omega_min=1e-12, max_viscosity_ratio=1e5, relaxation=0.7, tolerance=1e-6, k_transport=None,
                      omega_transport=None, k_solver=None, omega_solver=None):
        """turbulenceModel kOmega (before set_fields); k and omega then take boundary conditions."""
        cfg = KOmegaConfig(beta_star, beta, gamma, sigma_k, sigma_omega, k_min, omega_min, max_viscosity_ratio,
                           relaxation, tolerance, k_transport or options(), omega_transport or options(),
                           k_solver or solver_config("bcgs", "bjacobi", 1e-18, 1e-10, 1000),
                           omega_solver or solver_config("bcgs", "bjacobi", 1e-18, 1e-10, 1000))
        self._enable("komega", cfg)

    def enable_kepsilon(self, c_mu=0.09, c1=1.44, c2=1.92, sigma_k=1.0, sigma_epsilon=1.3, k_min=1e-12,
                        epsilon_min=1e-12, relaxation=0.7, tolerance=1e-6, k_transport=None, epsilon_transport=None,
                        k_solver=None, epsilon_solver=None):
        """turbulenceModel kEpsilon (before set_fields); k and epsilon then take boundary conditions."""
        cfg = KEpsilonConfig(c_mu, c1, c2, sigma_k, sigma_epsilon, k_min, epsilon_min, relaxation, tolerance,
                             k_transport or options(), epsilon_transport or options(),
                             k_solver or solver_config("bcgs", "bjacobi", 1e-18, 1e-10, 1000),
                             epsilon_solver or solver_config("bcgs", "bjacobi", 1e-18, 1e-10, 1000))
        self._enable("kepsilon", cfg)

    def enable_spalart_allmaras(self, cb1=0.1355, cb2=0.622, sigma=2.0 / 3.0, kappa=0.41, cw1=0.0, cw2=0.3, cw3=2.0,
                                cv1=7.1, ct3=1.2, ct4=0.5, nu_tilda_min=1e-14, wall_distance_min=1e-12,
                                relaxation=0.7, tolerance=1e-6, nu_tilda_transport=None, nu_tilda_solver=None):
        """turbulenceModel SA (before set_fields); "nuTilda" then takes boundary conditions and the wall
        distance comes from set_wall_distance.  cw1 <= 0 takes cb1/kappa^2 + (1 + cb2)/sigma."""
        cfg = SaConfig(cb1, cb2, sigma, kappa, cw1, cw2, cw3, cv1, ct3, ct4, nu_tilda_min, wall_distance_min,
                       relaxation, tolerance, nu_tilda_transport or options(),
                       nu_tilda_solver or solver_config("bcgs", "bjacobi", 1e-18, 1e-10, 1000))
        self._enable("spalart_allmaras", cfg)
        self._one_equation = True

    def set_wall_distance(self, d):
        """The wall distance of every cell (an input of the Spalart-Allmaras model, as in the reference)."""
        check(self._fn("set_wall_distance")(self.h, ptr(f64(d))), self.mesh.ctx.h)

    def set_turbulence_fields(self, k, second):
        """Initial k and omega / epsilon; k is None for Spalart-Allmaras, whose field is nuTilda."""
        kp = None if k is None else ptr(f64(k))
        check(self._fn("set_turbulence_fields")(self.h, kp, ptr(f64(second))), self.mesh.ctx.h)

    def turbulence_fields(self):
        """(k, second transported field, mut); k is None for Spalart-Allmaras."""
        n = self.mesh.n_cells
        one = getattr(self, "_one_equation", False)
        k, w, mut = (None if one else np.zeros(n)), np.zeros(n), np.zeros(n)
        check(self._fn("get_turbulence_fields")(self.h, None if one else ptr(k), ptr(w), ptr(mut)),
              self.mesh.ctx.h)
        return k, w, mut


class Simple(_TurbulenceModels):
    """Steady SIMPLE on the device (bsg_simple), simple/main.cpp:11-131."""
    _prefix = "bsg_simple_"

    def __init__(self, mesh: Mesh, rho=1.0, mu=0.01, alpha_u=0.7, alpha_p=0.3, non_orthogonal_corrections=1,
                 continuity_tolerance=1e-8, velocity_tolerance=1e-7, momentum_tolerance=1e-6,
                 pressure_tolerance=1e-6, momentum=None, pressure=None, momentum_solver=None, pressure_solver=None):
        self.mesh = mesh
        cfg = SimpleConfig(rho, mu, alpha_u, alpha_p, non_orthogonal_corrections, continuity_tolerance,
                           velocity_tolerance, momentum_tolerance, pressure_tolerance,
                           momentum or options(), pressure or options(),
                           momentum_solver or solver_config("bcgs", "bjacobi", 1e-14, 1e-10),
                           pressure_solver or solver_config("cg", "jacobi", 1e-14, 1e-10, 5000))
        h = C.c_void_p()
        check(lib().bsg_simple_create(mesh.h, C.byref(cfg), C.byref(h)), mesh.ctx.h)
        self.h = h

    def set_boundary(self, field: str, patch: int, kind: str, value=0.0):
        v = f64(np.broadcast_to(np.asarray(value, np.float64), (3,)) if np.ndim(value) == 0 else
                np.pad(np.asarray(value, np.float64), (0, 3 - len(value))))
        check(lib().bsg_simple_set_boundary(self.h, field.encode(), patch, BC[kind], ptr(v)), self.mesh.ctx.h)

    def set_fields(self, U, p):
        check(lib().bsg_simple_set_fields(self.h, ptr(f64(U)), ptr(f64(p))), self.mesh.ctx.h)

    def set_flux(self, phi):
        check(lib().bsg_simple_set_flux(self.h, ptr(f64(phi))), self.mesh.ctx.h)

    def load_state(self, U, p, phi):
        """Copy host U, p, phi in between outer iterations (no restart)."""
        check(lib().bsg_simple_load_state(self.h, ptr(U), ptr(p), ptr(phi)), self.mesh.ctx.h)

    def fields_into(self, U, p, phi):
        """Download U, p, phi into caller-provided (pinned) arrays."""
        check(lib().bsg_simple_get_fields(self.h, ptr(U), ptr(p), ptr(phi)), self.mesh.ctx.h)

    def iterate(self, max_iterations: int) -> SimpleReport:
        r = SimpleReport()
        check(lib().bsg_simple_iterate(self.h, max_iterations, C.byref(r)), self.mesh.ctx.h)
        return r

    def set_segments(self, cell_offsets, viscosity):
        """Block-diagonal batch: case k owns cells [cell_offsets[k], cell_offsets[k+1]) of a mesh
        made by meshgen.concatenate, with dynamic viscosity viscosity[k] (before set_fields)."""
        off = np.ascontiguousarray(cell_offsets, dtype=np.int32)
        mu = f64(viscosity)
        check(lib().bsg_simple_set_segments(self.h, len(mu), ptr(off), ptr(mu)), self.mesh.ctx.h)

    def segment_report(self, k: int) -> SimpleReport:
        r = SimpleReport()
        check(lib().bsg_simple_segment_report(self.h, k, C.byref(r)), self.mesh.ctx.h)
        return r

    def fields(self):
        m = self.mesh
        U, p, phi = np.zeros((m.n_cells, 3)), np.zeros(m.n_cells), np.zeros(m.n_faces)
        check(lib().bsg_simple_get_fields(self.h, ptr(U), ptr(p), ptr(phi)), m.ctx.h)
        return U, p, phi

    def close(self):
        if self.h:
            lib().bsg_simple_destroy(self.h)
            self.h = None


class Piso(_TurbulenceModels):
    """Transient PISO on the device (bsg_piso), piso/main.cpp:60-301.  A turbulence model is enabled
    with enable_komega / enable_kepsilon / enable_spalart_allmaras after set_turbulence_controls
    (runPiso's turbulenceCoupling, turbulenceMaxIterations, turbulenceCorrectors)."""
    _prefix = "bsg_piso_"
    _controls = None

    def set_turbulence_controls(self, coupling="iterated", max_iterations=1000, correctors=0):
        self._controls = PisoTurbulenceControls({"iterated": 0, "segregated": 1}[coupling], max_iterations,
                                                correctors)

    def _enable(self, model, cfg):
        ctl = self._controls or PisoTurbulenceControls(0, 1000, 0)
        check(self._fn("enable_" + model)(self.h, C.byref(cfg), C.byref(ctl)), self.mesh.ctx.h)

    def __init__(self, mesh: Mesh, rho=1.0, mu=0.01, alpha_u=1.0, max_iterations=1, correctors=2,
                 max_correctors=None, coupling_tolerance=None, non_orthogonal_corrections=1,
                 continuity_tolerance=1e-8, velocity_tolerance=1e-7, momentum_tolerance=1e-6, pressure_tolerance=1e-6,
                 time="bdf2", start_time=0.0, end_time=1.0, delta_t=1e-3, momentum=None, pressure=None,
                 momentum_solver=None, pressure_solver=None):
        self.mesh = mesh
        cfg = PisoConfig(rho, mu, alpha_u, max_iterations, correctors, max_correctors or correctors,
                         coupling_tolerance or 0.0, non_orthogonal_corrections, continuity_tolerance,
                         velocity_tolerance, momentum_tolerance, pressure_tolerance,
                         {"steady": 0, "euler": 1, "bdf2": 2}[time.lower()], start_time, end_time, delta_t,
                         momentum or options(), pressure or options(),
                         momentum_solver or solver_config("bcgs", "bjacobi", 1e-14, 1e-10),
                         pressure_solver or solver_config("cg", "hypre", 1e-14, 1e-10, 5000))
        h = C.c_void_p()
        check(lib().bsg_piso_create(mesh.h, C.byref(cfg), C.byref(h)), mesh.ctx.h)
        self.h = h

    def set_boundary(self, field: str, patch: int, kind: str, value=0.0):
        v = f64(np.broadcast_to(np.asarray(value, np.float64), (3,)) if np.ndim(value) == 0 else
                np.pad(np.asarray(value, np.float64), (0, 3 - len(value))))
        check(lib().bsg_piso_set_boundary(self.h, field.encode(), patch, BC[kind], ptr(v)), self.mesh.ctx.h)

    def initialize_potential_flow(self, initial_non_orthogonal_corrections=-1):
        """initializePotentialFlow 1: a potential-flow start before the first step (before set_fields)."""
        check(lib().bsg_piso_initialize_potential_flow(self.h, initial_non_orthogonal_corrections), self.mesh.ctx.h)

    def set_fields(self, U, p):
        check(lib().bsg_piso_set_fields(self.h, ptr(f64(U)), ptr(f64(p))), self.mesh.ctx.h)

    def advance(self, steps: int) -> PisoReport:
        r = PisoReport()
        check(lib().bsg_piso_advance(self.h, steps, C.byref(r)), self.mesh.ctx.h)
        return r

    def fields(self):
        m = self.mesh
        U, p, phi = np.zeros((m.n_cells, 3)), np.zeros(m.n_cells), np.zeros(m.n_faces)
        check(lib().bsg_piso_get_fields(self.h, ptr(U), ptr(p), ptr(phi)), m.ctx.h)
        return U, p, phi

    def close(self):
        if self.h:
            lib().bsg_piso_destroy(self.h)
            self.h = None


def write_results(time_directory: str, time_name: str, poly, fields: dict):
    """Write cell fields in the reference's result format (bsg_write_results): one CSV per field
    under <time_directory>/rank-0000 with metadata.bs and mesh.geometry.  `fields` maps a name
    to an (n_cells,) or (n_cells, 3) or (n_cells, 9) array in the caller's cell numbering."""
    off, ids = poly.flat()
    names = list(fields)
    arrays = [f64(np.asarray(fields[k], dtype=np.float64).reshape(poly.n_cells, -1)) for k in names]
    comps = np.array([a.shape[1] for a in arrays], dtype=np.int32)
    name_arr = (C.c_char_p * len(names))(*[n.encode() for n in names])
    val_arr = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    verts = f64(poly.vertices)
    owner, nbr, patch = i32(poly.owner), i32(poly.neighbour), i32(poly.patch)
    off, ids = i32(off), i32(ids)
    check(lib().bsg_write_results(str(time_directory).encode(), time_name.encode(), len(verts), ptr(verts),
                                  len(owner), ptr(off), ptr(ids), ptr(owner), ptr(nbr), ptr(patch),
                                  len(poly.patch_names), len(names), name_arr, ptr(comps), val_arr))
