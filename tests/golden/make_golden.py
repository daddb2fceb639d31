"""Generate golden fixtures from the reference's own finite-volume sources.

    python tests/golden/make_golden.py

Requires oracle/_ref/babelsim-oracle (built by `make -C oracle/ref`, which
compiles the reference sources in place).  For each case it writes a BabelSim
case directory, runs the reference's unmodified SIMPLE loop for k = 1..K outer
iterations (one run per k, so the state after every iteration is captured) and
to convergence, and stores in tests/golden/<case>.npz:

* the mesh (vertices, face rings, owner/neighbour/patch) and the geometry the
  reference computed from it;
* the assembled LDU systems of iteration K (momentum after relax/scale, each
  pressure-correction system) as handed to the linear-solver backend;
* U, p, phi after every iteration k <= K and at convergence.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from babelsim_b200 import meshgen  # noqa: E402
from oracle import refdata  # noqa: E402

ORACLE = os.path.join(ROOT, "oracle", "_ref", "babelsim-oracle")
OUT = os.path.dirname(os.path.abspath(__file__))

BC_TEXT = {"fixedValue": "fixedValue", "zeroGradient": "zeroGradient", "symmetry": "symmetry",
           "fixedGradient": "fixedGradient", "inletOutlet": "inletOutlet"}


def vec(v):
    return f"({v[0]!r} {v[1]!r} {v[2]!r})"


def write_case(path, mesh, U_bcs, p_bcs, methods, solution, physics, solver="simple", time="steady",
               control=(0.0, 0.0, 1.0), extra_fields=(), internal=None):
    """A BabelSim case directory.  `internal` maps U/p to an `internal` specification line
    (e.g. "file <results-dir>") instead of a zero uniform initial value."""
    internal = internal or {}
    os.makedirs(os.path.join(path, "mesh"), exist_ok=True)
    os.makedirs(os.path.join(path, "fields", "initial"), exist_ok=True)
    os.makedirs(os.path.join(path, "numerics"), exist_ok=True)
    os.makedirs(os.path.join(path, "physics"), exist_ok=True)
    meshgen.write_mesh(os.path.join(path, "mesh", "case.mesh"), mesh)
    with open(os.path.join(path, "case.bs"), "w") as f:
        f.write(f"solver {solver}\nmesh mesh/case.mesh\nfields fields/initial\nphysics physics/simple.bs\n"
                "methods numerics/methods.bs\nsolution numerics/solution.bs\ncontrol control.bs\noutput output.bs\n")
    with open(os.path.join(path, "control.bs"), "w") as f:
        f.write("startTime %r\nendTime %r\ndeltaT %r\n" % tuple(control))
    with open(os.path.join(path, "output.bs"), "w") as f:
        f.write("directory results\ntimeName final\n")
    with open(os.path.join(path, "physics", "simple.bs"), "w") as f:
        f.write("".join(f"{k} {v!r}\n" for k, v in physics.items()))
    with open(os.path.join(path, "numerics", "methods.bs"), "w") as f:
        f.write(f"time {time}\n")
        for eq, opts in methods.items():
            for k, v in opts.items():
                f.write(f"equation.{eq}.{k} {v}\n")
    with open(os.path.join(path, "numerics", "solution.bs"), "w") as f:
        f.write("".join(f"{k} {v}\n" for k, v in solution.items()))

    internal_spec = internal

    def field(name, kind, bcs, internal=0.0):
        spec = internal_spec.get(name) if internal_spec else None
        lines = [f"field {name}", "{", f"    type {kind}", "    location cell",
                 "    internal " + (spec if spec else ("uniform (0 0 0)" if kind == "vector" else f"uniform ({internal!r})")),
                 "    boundary", "    {"]
        for patch, (t, v) in zip(mesh.patch_names, bcs):
            if t in ("zeroGradient", "symmetry"):
                lines.append(f"        {patch} {{ type {t} }}")
            else:
                val = vec(v) if kind == "vector" else f"({v!r})"
                lines.append(f"        {patch} {{ type {t} value {val} }}")
        lines += ["    }", "}"]
        with open(os.path.join(path, "fields", "initial", f"{name}.field"), "w") as f:
            f.write("\n".join(lines) + "\n")
    field("U", "vector", U_bcs)
    field("p", "scalar", p_bcs)
    for name, internal, bcs in extra_fields:
        field(name, "scalar", bcs, internal)


def run(case_dir, iterations, dump=False):
    sol = os.path.join(case_dir, "numerics", "solution.bs")
    text = open(sol).read().splitlines()
    text = [ln for ln in text if not ln.startswith("maxIterations ")] + [f"maxIterations {iterations}"]
    open(sol, "w").write("\n".join(text) + "\n")
    out = tempfile.mkdtemp(prefix="bsg_golden_")
    env = dict(os.environ)
    if dump:
        os.makedirs(os.path.join(out, "dump"))
        env["BABELSIM_ORACLE_DUMP"] = os.path.join(out, "dump")
    res = subprocess.run([ORACLE, case_dir, out], env=env, capture_output=True, text=True)
    if res.returncode not in (0, 2):
        raise RuntimeError(res.stderr)
    fields = refdata.read_records(os.path.join(out, "fields.bin"))
    geo = refdata.read_records(os.path.join(out, "geometry.bin"))
    info = json.load(open(os.path.join(out, "run.json")))
    systems = refdata.read_systems(os.path.join(out, "dump")) if dump else []
    shutil.rmtree(out)
    return fields, geo, info, systems


def make(name, mesh, U_bcs, p_bcs, methods, solution, physics, K, converge_iterations=None):
    work = tempfile.mkdtemp(prefix=f"bsg_case_{name}_")
    write_case(work, mesh, U_bcs, p_bcs, methods, solution, physics)
    data = {}
    offsets, ids = mesh.flat()
    data["mesh_vertices"] = mesh.vertices
    data["mesh_offsets"] = np.asarray(offsets, dtype=np.int32)
    data["mesh_ids"] = np.asarray(ids, dtype=np.int32)
    data["mesh_owner"], data["mesh_neighbour"], data["mesh_patch"] = mesh.owner, mesh.neighbour, mesh.patch
    for k in range(1, K + 1):
        fields, geo, info, systems = run(work, k, dump=(k == K))
        data[f"U_{k}"] = fields["U"].reshape(-1, 3)
        data[f"p_{k}"] = fields["p"]
        data[f"phi_{k}"] = fields["phi"]
    for key, arr in geo.items():
        data["geo_" + key] = arr
    for j, s in enumerate(systems):
        for key in ("diag", "upper", "lower", "source", "before", "after"):
            data[f"sys{j}_{key}"] = s[key]
        data[f"sys{j}_meta"] = np.array([s["status"], s["iterations"]])
        data[f"sys{j}_identity"] = np.array(s["identity"])
    data["n_systems_last"] = np.array(len(systems))
    if converge_iterations:
        fields, _, info, _ = run(work, converge_iterations)
        data["U_conv"], data["p_conv"], data["phi_conv"] = fields["U"].reshape(-1, 3), fields["p"], fields["phi"]
        data["conv_info"] = np.array([info["status"], info["reported_iteration_intervals"] + 1])
    meta = dict(patch_names=mesh.patch_names, patch_kinds=mesh.patch_kinds, U_bcs=[(t, list(map(float, v)))
                for t, v in U_bcs], p_bcs=[(t, float(v)) for t, v in p_bcs], methods=methods,
                solution=solution, physics=physics, K=K)
    data["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **data)
    shutil.rmtree(work)
    print(name, "written", {k: v.shape for k, v in data.items() if k.startswith(("U_", "sys0_diag"))})


def cavity_bcs(lid=(1.0, 0.0, 0.0)):
    U = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", lid), ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    p = [("zeroGradient", 0.0)] * 4 + [("symmetry", 0.0)] * 2
    return U, p


def config1_solution(p_rtol=1e-10):
    return {"velocityRelaxation": 0.7, "pressureRelaxation": 0.3, "continuityTolerance": 1e-6,
            "velocityTolerance": 1e-6, "momentumTolerance": 1e-6, "pressureCorrectionTolerance": 1e-6,
            "nonOrthogonalCorrections": 2,
            "equation.momentum.kspType": "bcgs", "equation.momentum.pcType": "bjacobi",
            "equation.momentum.absoluteTolerance": 1e-15, "equation.momentum.relativeTolerance": 1e-12,
            "equation.momentum.maxIterations": 2000,
            "equation.pressureCorrection.kspType": "cg", "equation.pressureCorrection.pcType": "hypre",
            "equation.pressureCorrection.absoluteTolerance": 1e-15,
            "equation.pressureCorrection.relativeTolerance": p_rtol,
            "equation.pressureCorrection.maxIterations": 20000}


def methods(conv="upwind", grad="greenGauss", diff="orthogonal"):
    o = dict(interpolation="linear", gradient=grad, convection=conv, diffusion=diff)
    return {"momentum": o, "pressureCorrection": o}


def make_piso(name, mesh, U_bcs, p_bcs, methods, solution, physics, time, start, dt, ends, extra_fields=(),
              internal=None, files=None, turbulence_keys=(), extra_meta=None, arrays=None):
    """Transient fixture: the reference's runPiso to each end time in `ends` (one run per step).  With a
    turbulence model: `extra_fields` / `internal` / `files` give its input fields and `turbulence_keys`
    the fields stored after each step."""
    work = tempfile.mkdtemp(prefix=f"bsg_case_{name}_")
    data = dict(arrays or {})
    offsets = np.concatenate([[0], np.cumsum([len(f) for f in mesh.faces])]).astype(np.int32)
    data["mesh_vertices"] = mesh.vertices
    data["mesh_offsets"] = offsets
    data["mesh_ids"] = np.concatenate(mesh.faces).astype(np.int32)
    data["mesh_owner"], data["mesh_neighbour"], data["mesh_patch"] = mesh.owner, mesh.neighbour, mesh.patch
    for k, end in enumerate(ends, start=1):
        write_case(work, mesh, U_bcs, p_bcs, methods, solution, physics, solver="piso", time=time,
                   control=(start, end, dt), extra_fields=extra_fields, internal=internal)
        for fname, text in (files or {}).items():
            with open(os.path.join(work, "fields", "initial", fname), "w") as f:
                f.write(text)
        fields, geo, info, _ = run(work, solution.get("maxIterations", 1))
        if info["status"] != 0:
            raise RuntimeError(f"{name}: reference PISO did not complete step {k}: {info}")
        data[f"U_{k}"] = fields["U"].reshape(-1, 3)
        data[f"p_{k}"] = fields["p"]
        data[f"phi_{k}"] = fields["phi"]
        for key in turbulence_keys:
            data[f"{key}_{k}"] = fields[key]
    for key, arr in geo.items():
        data["geo_" + key] = arr
    meta = dict(patch_names=mesh.patch_names, patch_kinds=mesh.patch_kinds, U_bcs=[(t, list(map(float, v)))
                for t, v in U_bcs], p_bcs=[(t, float(v)) for t, v in p_bcs], methods=methods,
                solution=solution, physics=physics, K=len(ends), time=time, start=start, dt=dt, ends=list(ends))
    meta.update(extra_meta or {})
    data["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **data)
    shutil.rmtree(work)
    print(name, "written", len(ends), "steps")


def make_rans(name, mesh, U_bcs, p_bcs, k_field, w_field, methods, solution, physics, K, second="omega"):
    """Steady SIMPLE with the reference's k-omega (or k-epsilon) model: U, p, phi, k and the second
    transported field after iterations 1..K (stored under omega_* for both models)."""
    work = tempfile.mkdtemp(prefix=f"bsg_case_{name}_")
    write_case(work, mesh, U_bcs, p_bcs, methods, solution, physics,
               extra_fields=[("k",) + tuple(k_field), (second,) + tuple(w_field)])
    data = {}
    offsets, ids = mesh.flat()
    data["mesh_vertices"] = mesh.vertices
    data["mesh_offsets"] = np.asarray(offsets, dtype=np.int32)
    data["mesh_ids"] = np.asarray(ids, dtype=np.int32)
    data["mesh_owner"], data["mesh_neighbour"], data["mesh_patch"] = mesh.owner, mesh.neighbour, mesh.patch
    for k in range(1, K + 1):
        fields, geo, info, _ = run(work, k)
        data[f"U_{k}"] = fields["U"].reshape(-1, 3)
        for key in ("p", "phi", "k", second, "mut", "muEffective"):
            data[f"{'omega' if key == second else key}_{k}"] = fields[key]
    for key, arr in geo.items():
        data["geo_" + key] = arr
    meta = dict(patch_names=mesh.patch_names, patch_kinds=mesh.patch_kinds,
                U_bcs=[(t, list(map(float, v))) for t, v in U_bcs], p_bcs=[(t, float(v)) for t, v in p_bcs],
                k_internal=k_field[0], k_bcs=[(t, float(v)) for t, v in k_field[1]],
                omega_internal=w_field[0], omega_bcs=[(t, float(v)) for t, v in w_field[1]],
                methods=methods, solution=solution, physics=physics, K=K, second=second)
    data["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **data)
    shutil.rmtree(work)
    print(name, "written", K, "iterations")


def rans_methods(conv="upwind", grad="greenGauss", diff="orthogonal", turb_conv="upwind", second="omega"):
    o = dict(interpolation="linear", gradient=grad, convection=conv, diffusion=diff)
    t = dict(o, convection=turb_conv)
    return {"momentum": o, "pressureCorrection": o, "kTransport": t, f"{second}Transport": t}


def rans_solution(second="omega"):
    sol = config1_solution(1e-12)
    sol.update({"turbulenceRelaxation": 0.7, "turbulenceTolerance": 1e-6})
    for eq in ("kTransport", f"{second}Transport"):
        sol.update({f"equation.{eq}.kspType": "bcgs", f"equation.{eq}.pcType": "bjacobi",
                    f"equation.{eq}.absoluteTolerance": 1e-18, f"equation.{eq}.relativeTolerance": 1e-12,
                    f"equation.{eq}.maxIterations": 2000})
    return sol


def main_rans():
    komega = {"density": 1.0, "dynamicViscosity": 0.001, "turbulenceModel": "kOmega", "kOmegaBetaStar": 0.09,
              "kOmegaBeta": 0.075, "kOmegaGamma": 5.0 / 9.0, "kOmegaSigmaK": 0.5, "kOmegaSigmaOmega": 0.5,
              "kMin": 1e-12, "omegaMin": 1e-10, "maxTurbulentViscosityRatio": 1e5}
    # channel: inlet / outlet / two walls, one cell thick
    ch = meshgen.hex_box(16, 8, 1, hi=(4.0, 1.0, 0.25),
                         names=["inlet", "outlet", "lower", "upper", "front", "back"],
                         kinds=["inlet", "outlet", "wall", "wall", "symmetry", "symmetry"])
    U = [("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0)), ("fixedValue", (0.0, 0.0, 0.0)),
         ("fixedValue", (0.0, 0.0, 0.0)), ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    p = [("zeroGradient", 0.0), ("fixedValue", 0.0), ("zeroGradient", 0.0), ("zeroGradient", 0.0),
         ("symmetry", 0.0), ("symmetry", 0.0)]
    kb = [("fixedValue", 3.75e-3), ("zeroGradient", 0.0), ("fixedValue", 1e-12), ("fixedValue", 1e-12),
          ("symmetry", 0.0), ("symmetry", 0.0)]
    wb = [("fixedValue", 2.0), ("zeroGradient", 0.0), ("fixedValue", 800.0), ("fixedValue", 800.0),
          ("symmetry", 0.0), ("symmetry", 0.0)]
    make_rans("komega_channel", ch, U, p, (3.75e-3, kb), (2.0, wb), rans_methods("linearUpwind"), rans_solution(),
              komega, K=4)
    # warped box: lid, least squares, corrected diffusion, 2 non-orthogonal correctors
    Uw = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", (1.0, 0.0, 0.0))] + [("fixedValue", (0.0, 0.0, 0.0))] * 2
    pw = [("zeroGradient", 0.0)] * 6
    kw = [("fixedValue", 1e-12)] * 6
    ww = [("fixedValue", 500.0)] * 6
    make_rans("komega_warped5", meshgen.warped_box(5), Uw, pw, (1e-3, kw), (5.0, ww),
              rans_methods("linearUpwind", "leastSquares", "corrected"), rans_solution(), komega, K=3)
    # standard k-epsilon in the same channel
    keps = {"density": 1.0, "dynamicViscosity": 0.001, "turbulenceModel": "kEpsilon", "kEpsilonCmu": 0.09,
            "kEpsilonC1": 1.44, "kEpsilonC2": 1.92, "kEpsilonSigmaK": 1.0, "kEpsilonSigmaEpsilon": 1.3,
            "kMin": 1e-12, "epsilonMin": 1e-12}
    eb = [("fixedValue", 2.0e-4), ("zeroGradient", 0.0), ("fixedValue", 1e-10), ("fixedValue", 1e-10),
          ("symmetry", 0.0), ("symmetry", 0.0)]
    make_rans("kepsilon_channel", ch, U, p, (3.75e-3, kb), (2.0e-4, eb), rans_methods("linearUpwind", second="epsilon"),
              rans_solution("epsilon"), keps, K=4, second="epsilon")


def make_sa(name, mesh, U_bcs, p_bcs, nt_field, wall_distance, methods, solution, physics, K):
    """Steady SIMPLE with the reference's Spalart-Allmaras model: U, p, phi, nuTilda, mut after iterations
    1..K.  The wall distance is a given cell field (the reference reads it, it does not compute it),
    written as a file-backed internal value."""
    work = tempfile.mkdtemp(prefix=f"bsg_case_{name}_")
    write_case(work, mesh, U_bcs, p_bcs, methods, solution, physics,
               extra_fields=[("nuTilda",) + tuple(nt_field),
                             ("wallDistance", 0.0, [("zeroGradient", 0.0)] * len(mesh.patch_names))],
               internal={"wallDistance": "file wallDistance.data"})
    with open(os.path.join(work, "fields", "initial", "wallDistance.data"), "w") as f:
        f.write("".join(f"{i} {d!r}\n" for i, d in enumerate(map(float, wall_distance))))
    data = {}
    offsets, ids = mesh.flat()
    data["mesh_vertices"] = mesh.vertices
    data["mesh_offsets"] = np.asarray(offsets, dtype=np.int32)
    data["mesh_ids"] = np.asarray(ids, dtype=np.int32)
    data["mesh_owner"], data["mesh_neighbour"], data["mesh_patch"] = mesh.owner, mesh.neighbour, mesh.patch
    data["wall_distance"] = np.asarray(wall_distance, dtype=np.float64)
    for k in range(1, K + 1):
        fields, geo, info, _ = run(work, k)
        data[f"U_{k}"] = fields["U"].reshape(-1, 3)
        for key in ("p", "phi", "nuTilda", "mut", "muEffective"):
            data[f"{key}_{k}"] = fields[key]
    for key, arr in geo.items():
        data["geo_" + key] = arr
    meta = dict(patch_names=mesh.patch_names, patch_kinds=mesh.patch_kinds,
                U_bcs=[(t, list(map(float, v))) for t, v in U_bcs], p_bcs=[(t, float(v)) for t, v in p_bcs],
                nuTilda_internal=nt_field[0], nuTilda_bcs=[(t, float(v)) for t, v in nt_field[1]],
                methods=methods, solution=solution, physics=physics, K=K)
    data["meta"] = np.array(json.dumps(meta))
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **data)
    shutil.rmtree(work)
    print(name, "written", K, "iterations")


def _cell_centres(mesh):
    from oracle import geometry
    return geometry.compute_geometry(geometry.PolyMesh(mesh.vertices, mesh.rings(), mesh.owner, mesh.neighbour,
                                                       mesh.patch, mesh.patch_names, mesh.patch_kinds)).xc


def main_sa():
    sa = {"density": 1.0, "dynamicViscosity": 0.001, "turbulenceModel": "SA", "saNuTildaMin": 1e-14,
          "saWallDistanceMin": 1e-12, "saCb1": 0.1355, "saCb2": 0.622, "saSigma": 2.0 / 3.0, "saKappa": 0.41,
          "saCw2": 0.3, "saCw3": 2.0, "saCv1": 7.1, "saCt3": 1.2, "saCt4": 0.5}

    def methods_sa(conv="upwind", grad="greenGauss", diff="orthogonal"):
        o = dict(interpolation="linear", gradient=grad, convection=conv, diffusion=diff)
        return {"momentum": o, "pressureCorrection": o, "nuTildaTransport": dict(o, convection="upwind")}

    def solution_sa():
        sol = config1_solution(1e-12)
        sol.update({"turbulenceRelaxation": 0.7, "turbulenceTolerance": 1e-6,
                    "equation.nuTildaTransport.kspType": "bcgs", "equation.nuTildaTransport.pcType": "bjacobi",
                    "equation.nuTildaTransport.absoluteTolerance": 1e-18,
                    "equation.nuTildaTransport.relativeTolerance": 1e-12,
                    "equation.nuTildaTransport.maxIterations": 2000})
        return sol
    ch = meshgen.hex_box(16, 8, 1, hi=(4.0, 1.0, 0.25),
                         names=["inlet", "outlet", "lower", "upper", "front", "back"],
                         kinds=["inlet", "outlet", "wall", "wall", "symmetry", "symmetry"])
    U = [("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0)), ("fixedValue", (0.0, 0.0, 0.0)),
         ("fixedValue", (0.0, 0.0, 0.0)), ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    p = [("zeroGradient", 0.0), ("fixedValue", 0.0), ("zeroGradient", 0.0), ("zeroGradient", 0.0),
         ("symmetry", 0.0), ("symmetry", 0.0)]
    ntb = [("fixedValue", 3e-3), ("zeroGradient", 0.0), ("fixedValue", 0.0), ("fixedValue", 0.0),
           ("symmetry", 0.0), ("symmetry", 0.0)]
    y = _cell_centres(ch)[:, 1]
    make_sa("sa_channel", ch, U, p, (3e-3, ntb), np.minimum(y, 1.0 - y), methods_sa("linearUpwind"),
            solution_sa(), sa, K=4)
    wb = meshgen.warped_box(5)
    Uw = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", (1.0, 0.0, 0.0))] + [("fixedValue", (0.0, 0.0, 0.0))] * 2
    pw = [("zeroGradient", 0.0)] * 6
    xc = _cell_centres(wb)
    d = np.minimum(np.minimum(xc, 1.0 - xc).min(axis=1), 1.0)
    make_sa("sa_warped5", wb, Uw, pw, (2e-3, [("fixedValue", 0.0)] * 6), d,
            methods_sa("linearUpwind", "leastSquares", "corrected"), solution_sa(), sa, K=3)


def piso_solution(n_correctors=2, non_orth=1, p_rtol=1e-12):
    return {"maxIterations": 1, "nCorrectors": n_correctors, "nonOrthogonalCorrections": non_orth,
            "velocityRelaxation": 1.0, "continuityTolerance": 1e-7, "velocityTolerance": 1e-7,
            "momentumTolerance": 1e-6, "pressureCorrectionTolerance": 1e-7,
            "equation.momentum.kspType": "bcgs", "equation.momentum.pcType": "bjacobi",
            "equation.momentum.absoluteTolerance": 1e-15, "equation.momentum.relativeTolerance": 1e-12,
            "equation.momentum.maxIterations": 2000,
            "equation.pressureCorrection.kspType": "cg", "equation.pressureCorrection.pcType": "hypre",
            "equation.pressureCorrection.absoluteTolerance": 1e-15,
            "equation.pressureCorrection.relativeTolerance": p_rtol,
            "equation.pressureCorrection.maxIterations": 20000}


def main_piso():
    U, p = cavity_bcs()
    # BDF2 lid cavity, 6 steps, the last one shortened (variable-step BDF2 weights)
    make_piso("piso_cavity12_bdf2", meshgen.cavity_2d(12), U, p, methods("linearUpwind"), piso_solution(2, 1),
              {"density": 1.0, "dynamicViscosity": 0.01}, "bdf2", 0.0, 0.05, [0.05, 0.1, 0.15, 0.2, 0.25, 0.27])
    # warped box, least squares + corrected diffusion, Euler, 3 correctors
    Uw = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", (1.0, 0.0, 0.0))] + [("fixedValue", (0.0, 0.0, 0.0))] * 2
    pw = [("zeroGradient", 0.0)] * 6
    make_piso("piso_warped5_euler", meshgen.warped_box(5), Uw, pw, methods("linearUpwind", "leastSquares", "corrected"),
              piso_solution(3, 2), {"density": 1.0, "dynamicViscosity": 0.01}, "euler", 0.0, 0.02,
              [0.02, 0.04, 0.06, 0.08])
    # flow past a cylinder on a small O-grid: inlet, outlet (p = 0), BDF2, corrected diffusion
    Uc = [("fixedValue", (0.0, 0.0, 0.0)), ("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0)),
          ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    pc = [("zeroGradient", 0.0), ("zeroGradient", 0.0), ("fixedValue", 0.0), ("symmetry", 0.0), ("symmetry", 0.0)]
    make_piso("piso_cylinder_ogrid", meshgen.cylinder_ogrid(48, 12, radius=6.0, growth=1.15), Uc, pc,
              methods("linearUpwind", "leastSquares", "corrected"), piso_solution(2, 1),
              {"density": 1.0, "dynamicViscosity": 0.01}, "bdf2", 0.0, 0.05, [0.05, 0.1, 0.15])


def main_piso_potential():
    """runPiso with initializePotentialFlow 1 (piso/main.cpp:123-146) on the inlet/outlet channel from
    rest: the first step starts from the potential-flow velocity and flux.  Corrected diffusion on the
    warped box exercises the non-orthogonal potential solves."""
    ch = meshgen.hex_box(16, 8, 1, hi=(4.0, 1.0, 0.25),
                         names=["inlet", "outlet", "lower", "upper", "front", "back"],
                         kinds=["inlet", "outlet", "wall", "wall", "symmetry", "symmetry"])
    U = [("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0)), ("fixedValue", (0.0, 0.0, 0.0)),
         ("fixedValue", (0.0, 0.0, 0.0)), ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    p = [("zeroGradient", 0.0), ("fixedValue", 0.0), ("zeroGradient", 0.0), ("zeroGradient", 0.0),
         ("symmetry", 0.0), ("symmetry", 0.0)]
    sol = dict(piso_solution(2, 1), initializePotentialFlow=1)
    make_piso("piso_potential_channel", ch, U, p, methods("linearUpwind"), sol,
              {"density": 1.0, "dynamicViscosity": 0.01}, "euler", 0.0, 0.05, [0.05, 0.1])
    wb = meshgen.warped_box(5, amplitude=0.08)
    Uw = [("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0))] + [("fixedValue", (0.0, 0.0, 0.0))] * 4
    pw = [("zeroGradient", 0.0), ("fixedValue", 0.0)] + [("zeroGradient", 0.0)] * 4
    sol = dict(piso_solution(2, 2), initializePotentialFlow=1, initialNonOrthogonalCorrections=3)
    make_piso("piso_potential_warped5", wb, Uw, pw, methods("linearUpwind", "leastSquares", "corrected"), sol,
              {"density": 1.0, "dynamicViscosity": 0.01}, "bdf2", 0.0, 0.02, [0.02, 0.04])


def main_piso_rans():
    """runPiso with a turbulence model (rans::load inside piso/main.cpp:98-121, transport after the
    correctors at every time level, 239-254): k-omega on the channel with BDF2, Spalart-Allmaras with Euler."""
    ch = meshgen.hex_box(16, 8, 1, hi=(4.0, 1.0, 0.25),
                         names=["inlet", "outlet", "lower", "upper", "front", "back"],
                         kinds=["inlet", "outlet", "wall", "wall", "symmetry", "symmetry"])
    U = [("fixedValue", (1.0, 0.0, 0.0)), ("zeroGradient", (0, 0, 0)), ("fixedValue", (0.0, 0.0, 0.0)),
         ("fixedValue", (0.0, 0.0, 0.0)), ("symmetry", (0, 0, 0)), ("symmetry", (0, 0, 0))]
    p = [("zeroGradient", 0.0), ("fixedValue", 0.0), ("zeroGradient", 0.0), ("zeroGradient", 0.0),
         ("symmetry", 0.0), ("symmetry", 0.0)]
    turb_sol = {"turbulenceRelaxation": 0.7, "turbulenceTolerance": 1e-6, "turbulenceMaxIterations": 400}

    def eq_controls(eq):
        return {f"equation.{eq}.kspType": "bcgs", f"equation.{eq}.pcType": "bjacobi",
                f"equation.{eq}.absoluteTolerance": 1e-18, f"equation.{eq}.relativeTolerance": 1e-12,
                f"equation.{eq}.maxIterations": 2000}
    # k-omega, BDF2
    komega = {"density": 1.0, "dynamicViscosity": 0.001, "turbulenceModel": "kOmega", "kOmegaBetaStar": 0.09,
              "kOmegaBeta": 0.075, "kOmegaGamma": 5.0 / 9.0, "kOmegaSigmaK": 0.5, "kOmegaSigmaOmega": 0.5,
              "kMin": 1e-12, "omegaMin": 1e-10, "maxTurbulentViscosityRatio": 1e5}
    kb = [("fixedValue", 3.75e-3), ("zeroGradient", 0.0), ("fixedValue", 1e-12), ("fixedValue", 1e-12),
          ("symmetry", 0.0), ("symmetry", 0.0)]
    wb = [("fixedValue", 2.0), ("zeroGradient", 0.0), ("fixedValue", 800.0), ("fixedValue", 800.0),
          ("symmetry", 0.0), ("symmetry", 0.0)]
    sol = dict(piso_solution(2, 1), **turb_sol, **eq_controls("kTransport"), **eq_controls("omegaTransport"))
    m = rans_methods("linearUpwind")
    make_piso("piso_komega_channel", ch, U, p, m, sol, komega, "bdf2", 0.0, 0.05, [0.05, 0.1, 0.15, 0.2],
              extra_fields=[("k", 3.75e-3, kb), ("omega", 2.0, wb)], turbulence_keys=("k", "omega", "mut"),
              extra_meta=dict(k_internal=3.75e-3, k_bcs=kb, omega_internal=2.0, omega_bcs=wb, second="omega"))
    # standard k-epsilon, BDF2
    keps = {"density": 1.0, "dynamicViscosity": 0.001, "turbulenceModel": "kEpsilon", "kEpsilonCmu": 0.09,
            "kEpsilonC1": 1.44, "kEpsilonC2": 1.92, "kEpsilonSigmaK": 1.0, "kEpsilonSigmaEpsilon": 1.3,
            "kMin": 1e-12, "epsilonMin": 1e-12}
    eb = [("fixedValue", 2.0e-4), ("zeroGradient", 0.0), ("fixedValue", 1e-10), ("fixedValue", 1e-10),
          ("symmetry", 0.0), ("symmetry", 0.0)]
    sol = dict(piso_solution(2, 1), **turb_sol, **eq_controls("kTransport"), **eq_controls("epsilonTransport"))
    make_piso("piso_kepsilon_channel", ch, U, p, rans_methods("linearUpwind", second="epsilon"), sol, keps, "bdf2",
              0.0, 0.05, [0.05, 0.1, 0.15], extra_fields=[("k", 3.75e-3, kb), ("epsilon", 2.0e-4, eb)],
              turbulence_keys=("k", "epsilon", "mut"),
              extra_meta=dict(k_internal=3.75e-3, k_bcs=kb, omega_internal=2.0e-4, omega_bcs=eb, second="epsilon"))
    # Spalart-Allmaras, Euler
    sa = {"density": 1.0, "dynamicViscosity": 0.001, "turbulenceModel": "SA", "saNuTildaMin": 1e-14,
          "saWallDistanceMin": 1e-12, "saCb1": 0.1355, "saCb2": 0.622, "saSigma": 2.0 / 3.0, "saKappa": 0.41,
          "saCw2": 0.3, "saCw3": 2.0, "saCv1": 7.1, "saCt3": 1.2, "saCt4": 0.5}
    ntb = [("fixedValue", 3e-3), ("zeroGradient", 0.0), ("fixedValue", 0.0), ("fixedValue", 0.0),
           ("symmetry", 0.0), ("symmetry", 0.0)]
    y = _cell_centres(ch)[:, 1]
    d = np.minimum(y, 1.0 - y)
    o = dict(interpolation="linear", gradient="greenGauss", convection="linearUpwind", diffusion="orthogonal")
    msa = {"momentum": o, "pressureCorrection": o, "nuTildaTransport": dict(o, convection="upwind")}
    sol = dict(piso_solution(2, 1), **turb_sol, **eq_controls("nuTildaTransport"))
    make_piso("piso_sa_channel", ch, U, p, msa, sol, sa, "euler", 0.0, 0.05, [0.05, 0.1, 0.15],
              extra_fields=[("nuTilda", 3e-3, ntb), ("wallDistance", 0.0, [("zeroGradient", 0.0)] * 6)],
              internal={"wallDistance": "file wallDistance.data"},
              files={"wallDistance.data": "".join(f"{i} {v!r}\n" for i, v in enumerate(map(float, d)))},
              turbulence_keys=("nuTilda", "mut"), arrays={"wall_distance": d},
              extra_meta=dict(nuTilda_internal=3e-3, nuTilda_bcs=ntb))


def main():
    if not os.path.exists(ORACLE):
        sys.exit(f"{ORACLE} missing: run `make -C oracle/ref` first")
    U, p = cavity_bcs()
    # config-1 settings on a 12x12x1 cavity (fast), 3 iterations + convergence
    make("cavity12_upwind", meshgen.cavity_2d(12), U, p, methods(), config1_solution(1e-12),
         {"density": 1.0, "dynamicViscosity": 0.01}, K=3, converge_iterations=2000)
    # the reference's own 64x64x1 cavity mesh with config-1 settings, converged
    # the reference checkout: $BABELSIM_REFERENCE, by default `reference` beside this repository
    ref_root = os.environ.get("BABELSIM_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
    ref_mesh = os.path.join(ref_root, "cases", "cavity", "mesh", "cavity.mesh")
    make("cavity64_config1", meshgen.read_mesh(ref_mesh), U, p, methods(), config1_solution(1e-12),
         {"density": 1.0, "dynamicViscosity": 0.01}, K=1, converge_iterations=5000)
    # non-orthogonal 3D: warped 5^3 box, LS gradient, corrected diffusion, linearUpwind, 2 correctors
    Uw = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", (1.0, 0.0, 0.0))] + [("fixedValue", (0.0, 0.0, 0.0))] * 2
    pw = [("zeroGradient", 0.0)] * 6
    make("warped5_corrected", meshgen.warped_box(5), Uw, pw, methods("linearUpwind", "leastSquares", "corrected"),
         config1_solution(1e-12), {"density": 1.0, "dynamicViscosity": 0.01}, K=3, converge_iterations=3000)


def config2_solution(rtol=1e-10):
    """The 1M-cell polyhedral cavity's solver controls: relaxation 0.7 / 0.3, 2 non-orthogonal
    correctors, momentum BiCGStab + block Jacobi and pressure CG + AMG, both to rtol 1e-10."""
    sol = config1_solution(rtol)
    sol["equation.momentum.relativeTolerance"] = rtol
    sol["equation.momentum.absoluteTolerance"] = 1e-15
    return sol


def main_voronoi():
    """Jittered-lattice Voronoi cubes (jitter 0.3h, seed 20261007: the generator and seed of the
    1M-cell bench workload) with its settings: lid u = 1 on plus_y, nu = 1e-3, linearUpwind
    convection, least-squares gradients, corrected diffusion, 2 non-orthogonal correctors."""
    lid = [("fixedValue", (0.0, 0.0, 0.0))] * 3 + [("fixedValue", (1.0, 0.0, 0.0))] + \
          [("fixedValue", (0.0, 0.0, 0.0))] * 2
    walls_p = [("zeroGradient", 0.0)] * 6
    m = methods("linearUpwind", "leastSquares", "corrected")
    make("voronoi8_config2", meshgen.voronoi_cube(8, 0.3, 20261007), lid, walls_p, m, config2_solution(),
         {"density": 1.0, "dynamicViscosity": 1e-3}, K=3, converge_iterations=4000)
    make("voronoi12_config2", meshgen.voronoi_cube(12, 0.3, 20261007), lid, walls_p, m, config2_solution(),
         {"density": 1.0, "dynamicViscosity": 1e-3}, K=2)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "voronoi":
        main_voronoi()
    elif len(sys.argv) > 1 and sys.argv[1] == "piso":
        main_piso()
    elif len(sys.argv) > 1 and sys.argv[1] == "rans":
        main_rans()
    elif len(sys.argv) > 1 and sys.argv[1] == "sa":
        main_sa()
    elif len(sys.argv) > 1 and sys.argv[1] == "piso_rans":
        main_piso_rans()
    elif len(sys.argv) > 1 and sys.argv[1] == "piso_potential":
        main_piso_potential()
    else:
        main()
        main_piso()
        main_rans()
        main_sa()
        main_piso_rans()
        main_piso_potential()
        main_voronoi()
