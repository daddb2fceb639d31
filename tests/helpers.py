"""Shared test helpers: golden fixtures, oracle set-up and the product's settings."""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from babelsim_b200 import meshgen  # noqa: E402
from oracle import fvm, geometry, piso, rans, simple  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
CASES = ["cavity12_upwind", "cavity64_config1", "warped5_corrected", "voronoi8_config2", "voronoi12_config2"]
# jittered-Voronoi polyhedral cubes with the 1M-cell bench workload's settings
VORONOI_CASES = ["voronoi8_config2", "voronoi12_config2"]
PISO_CASES = ["piso_cavity12_bdf2", "piso_warped5_euler", "piso_cylinder_ogrid"]
RANS_CASES = ["komega_channel", "komega_warped5"]
SA_CASES = ["sa_channel", "sa_warped5"]
PISO_RANS_CASES = ["piso_komega_channel", "piso_kepsilon_channel", "piso_sa_channel"]
PISO_POTENTIAL_CASES = ["piso_potential_channel", "piso_potential_warped5"]
GEO_KEYS = ["face_owner", "face_neighbour", "face_patch", "face_centres", "face_area_vectors", "face_areas",
            "face_normals", "face_owner_weights", "face_orthogonal_coefficients", "face_non_orthogonal",
            "face_skewness", "cell_centres", "cell_volumes", "orthogonal_geometry"]


class Golden:
    def __init__(self, name):
        self.name = name
        self.d = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.meta = json.loads(str(self.d["meta"]))
        off = self.d["mesh_offsets"]
        ids = self.d["mesh_ids"]
        faces = [ids[off[i]:off[i + 1]] for i in range(len(off) - 1)]
        self.poly = meshgen.PolyMesh(self.d["mesh_vertices"], faces, self.d["mesh_owner"], self.d["mesh_neighbour"],
                                     self.d["mesh_patch"], self.meta["patch_names"], self.meta["patch_kinds"])
        self.K = self.meta["K"]

    def __getitem__(self, k):
        return self.d[k]

    def ref_geometry(self):
        return {k: self.d["geo_" + k] for k in GEO_KEYS}

    def oracle_geometry(self):
        p = self.poly
        return geometry.compute_geometry(geometry.PolyMesh(p.vertices, p.faces, p.owner, p.neighbour, p.patch,
                                                           p.patch_names, p.patch_kinds))

    def U_bcs(self):
        return [(fvm.BC_NAMES[t], np.array(v, float)) for t, v in self.meta["U_bcs"]]

    def p_bcs(self):
        return [(fvm.BC_NAMES[t], float(v)) for t, v in self.meta["p_bcs"]]

    def systems(self):
        n = int(self.d["n_systems_last"])
        return [dict(identity=str(self.d[f"sys{j}_identity"]),
                     **{k: self.d[f"sys{j}_{k}"] for k in ("diag", "upper", "lower", "source", "before", "after")})
                for j in range(n)]

    def settings(self, **over) -> simple.SimpleSettings:
        sol = self.meta["solution"]
        m = self.meta["methods"]
        s = simple.SimpleSettings(rho=self.meta["physics"]["density"], mu=self.meta["physics"]["dynamicViscosity"],
                                  alpha_u=sol["velocityRelaxation"], alpha_p=sol["pressureRelaxation"],
                                  non_orthogonal_corrections=sol.get("nonOrthogonalCorrections", 1),
                                  mass_tolerance=sol["continuityTolerance"], velocity_tolerance=sol["velocityTolerance"],
                                  momentum_tolerance=sol["momentumTolerance"],
                                  pressure_tolerance=sol["pressureCorrectionTolerance"],
                                  momentum=dict(m["momentum"]), pressure=dict(m["pressureCorrection"]))
        for k, v in over.items():
            setattr(s, k, v)
        return s


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def rel_l2(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def ref_system_groups(g: Golden):
    """Split the dumped systems into per-iteration groups [momentum, pressure...]."""
    groups, cur = [], None
    for s in g.systems():
        if s["identity"] == "momentum":
            cur = dict(momentum=s, pressure=[])
            groups.append(cur)
        else:
            cur["pressure"].append(s)
    return groups


def piso_settings(g: "Golden", end_time=None) -> piso.PisoSettings:
    """PisoSettings of a transient fixture (the case written by tests/golden/make_golden.py)."""
    sol, m, phys = g.meta["solution"], g.meta["methods"], g.meta["physics"]
    return piso.PisoSettings(rho=phys["density"], mu=phys["dynamicViscosity"], alpha_u=sol["velocityRelaxation"],
                             max_iterations=sol["maxIterations"], correctors=sol["nCorrectors"],
                             non_orthogonal_corrections=sol["nonOrthogonalCorrections"],
                             mass_tolerance=sol["continuityTolerance"], velocity_tolerance=sol["velocityTolerance"],
                             momentum_tolerance=sol["momentumTolerance"],
                             pressure_tolerance=sol["pressureCorrectionTolerance"], time=g.meta["time"],
                             start_time=g.meta["start"], delta_t=g.meta["dt"],
                             end_time=g.meta["ends"][-1] if end_time is None else end_time,
                             momentum=m["momentum"], pressure=m["pressureCorrection"],
                             turbulence_max_iterations=sol.get("turbulenceMaxIterations", 1000),
                             initialize_potential_flow=bool(sol.get("initializePotentialFlow", 0)),
                             initial_non_orthogonal_corrections=sol.get("initialNonOrthogonalCorrections"))


def komega_constants(g: "Golden") -> rans.KOmegaConstants:
    ph, sol = g.meta["physics"], g.meta["solution"]
    return rans.KOmegaConstants(ph["kOmegaBetaStar"], ph["kOmegaBeta"], ph["kOmegaGamma"], ph["kOmegaSigmaK"],
                                ph["kOmegaSigmaOmega"], ph["kMin"], ph["omegaMin"], ph["maxTurbulentViscosityRatio"],
                                sol["turbulenceRelaxation"], sol["turbulenceTolerance"])


def komega_factory(g: "Golden"):
    """Model factory for oracle.simple.run_simple(turbulence=...) from a k-omega fixture."""
    ph, m = g.meta["physics"], g.meta["methods"]
    kb = [(fvm.BC_NAMES[t], v) for t, v in g.meta["k_bcs"]]
    wb = [(fvm.BC_NAMES[t], v) for t, v in g.meta["omega_bcs"]]

    def make(geo, phi0):
        k = fvm.Field(geo, np.full(geo.n_cells, g.meta["k_internal"]), kb)
        w = fvm.Field(geo, np.full(geo.n_cells, g.meta["omega_internal"]), wb)
        return rans.KOmega(geo, k, w, ph["density"], ph["dynamicViscosity"], komega_constants(g),
                           m["kTransport"], m["omegaTransport"], m["momentum"], phi0)
    return make


def kepsilon_factory(g: "Golden"):
    """Model factory for oracle.simple.run_simple(turbulence=...) from a k-epsilon fixture."""
    ph, sol, m = g.meta["physics"], g.meta["solution"], g.meta["methods"]
    c = rans.KEpsilonConstants(ph["kEpsilonCmu"], ph["kEpsilonC1"], ph["kEpsilonC2"], ph["kEpsilonSigmaK"],
                               ph["kEpsilonSigmaEpsilon"], ph["kMin"], ph["epsilonMin"], sol["turbulenceRelaxation"],
                               sol["turbulenceTolerance"])
    kb = [(fvm.BC_NAMES[t], v) for t, v in g.meta["k_bcs"]]
    eb = [(fvm.BC_NAMES[t], v) for t, v in g.meta["omega_bcs"]]

    def make(geo, phi0):
        k = fvm.Field(geo, np.full(geo.n_cells, g.meta["k_internal"]), kb)
        e = fvm.Field(geo, np.full(geo.n_cells, g.meta["omega_internal"]), eb)
        return rans.KEpsilon(geo, k, e, ph["density"], ph["dynamicViscosity"], c, m["kTransport"],
                             m["epsilonTransport"], m["momentum"], phi0)
    return make


def sa_constants(g: "Golden") -> rans.SpalartAllmarasConstants:
    ph, sol = g.meta["physics"], g.meta["solution"]
    return rans.SpalartAllmarasConstants(ph["saCb1"], ph["saCb2"], ph["saSigma"], ph["saKappa"], ph["saCw2"],
                                         ph["saCw3"], ph["saCv1"], ph["saCt3"], ph["saCt4"], None,
                                         ph["saNuTildaMin"], ph["saWallDistanceMin"], sol["turbulenceRelaxation"],
                                         sol["turbulenceTolerance"])


def sa_factory(g: "Golden"):
    """Model factory for oracle.simple.run_simple(turbulence=...) from a Spalart-Allmaras fixture."""
    ph, m = g.meta["physics"], g.meta["methods"]
    nb = [(fvm.BC_NAMES[t], v) for t, v in g.meta["nuTilda_bcs"]]

    def make(geo, phi0):
        nt = fvm.Field(geo, np.full(geo.n_cells, g.meta["nuTilda_internal"]), nb)
        return rans.SpalartAllmaras(geo, nt, g["wall_distance"], ph["density"], ph["dynamicViscosity"],
                                    sa_constants(g), m["nuTildaTransport"], m["momentum"], phi0)
    return make


def fields_at_reference_count(make_sim, n, target):
    """Run SIMPLE to convergence, then report the fields after exactly `target` outer
    iterations (the reference's count): continuing past an earlier convergence, or
    re-running when this run needed more.  Returns (report of the full run, U, p)."""
    sim = make_sim()
    sim.set_fields(np.zeros((n, 3)), np.zeros(n))
    r = sim.iterate(6000)
    if r.iterations > target:
        sim.close()
        sim = make_sim()
        sim.set_fields(np.zeros((n, 3)), np.zeros(n))
        sim.iterate(target)
    done = min(r.iterations, target)
    while done < target:
        done = sim.iterate(1).iterations
    U, p, _ = sim.fields()
    sim.close()
    return r, U, p


class ReferenceCounters:
    """PetscLinearSystem::updateMatrix / prepare / setup / solveRhs bookkeeping, one system."""

    def __init__(self, interval=8, growth=2.0):
        self.interval, self.growth = interval, growth
        self.matrix_updates = 0
        self.pc_matrix_update = 0
        self.setups = 0
        self.rhs_solves = 0
        self.fresh = 0
        self.setup_pending = True      # configure() (petsc_linear_system.cpp:190-194)
        self.force_rebuild = True

    def solve(self, changed, its, status):
        if changed:                    # updateMatrix: values differ
            self.matrix_updates += 1
            self.setup_pending = True
        rebuilt = False
        if self.setup_pending or self.force_rebuild:     # prepare
            reuse = (self.setups != 0 and not self.force_rebuild
                     and self.matrix_updates - self.pc_matrix_update < self.interval
                     and self.rhs_solves < self.interval)
            if not reuse:                                # setup(false)
                self.setups += 1
                self.pc_matrix_update = self.matrix_updates
                self.rhs_solves = 0
                self.fresh = 0
                rebuilt = True
            self.setup_pending = False
            self.force_rebuild = False
        if status == 0:                                  # solveRhs after a converged attempt
            if self.pc_matrix_update == self.matrix_updates:
                self.fresh = max(self.fresh, its)
            elif its > self.growth * max(self.fresh, 1):
                self.force_rebuild = True
        if its > 0:
            self.rhs_solves += 1
        return rebuilt

    def lagged(self):
        """After solve(): the solve ran with a preconditioner built for an older matrix."""
        return self.pc_matrix_update != self.matrix_updates
