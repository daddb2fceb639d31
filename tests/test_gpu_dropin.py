"""The reference's own program with its linear-system backend replaced by the B200 plugin.

oracle/_ref/babelsim-b200 is the reference's finite-volume sources and SIMPLE
loop, linked with babelsim_b200/integration/b200_compute_backend.cpp instead of
the PETSc units: every momentum and pressure solve goes through bsg_solve_ldu on
the GPU.  It must reach the reference's converged fields (golden fixtures).
The binary is built here from the reference sources and travels with the repo.
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from helpers import ROOT, Golden, rel_l2

pytestmark = pytest.mark.gpu
EXE = os.path.join(ROOT, "oracle", "_ref", "babelsim-b200")


def _run_program(g, max_iterations, never_converge=False):
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import write_case
    from oracle import refdata
    meta = g.meta
    work = tempfile.mkdtemp(prefix="bsg_dropin_")
    sol = dict(meta["solution"])
    sol["maxIterations"] = max_iterations
    if never_converge:
        # run exactly max_iterations outer iterations
        for key in ("continuityTolerance", "velocityTolerance", "momentumTolerance", "pressureCorrectionTolerance"):
            sol[key] = 1e-300
    write_case(work, g.poly, [(t, tuple(v)) for t, v in meta["U_bcs"]], [(t, v) for t, v in meta["p_bcs"]],
               meta["methods"], sol, meta["physics"])
    out = os.path.join(work, "out")
    res = subprocess.run([EXE, work, out], capture_output=True, text=True, timeout=600)
    assert res.returncode in ((0, 2) if never_converge else (0,)), res.stderr[-2000:]
    info = json.load(open(os.path.join(out, "run.json")))
    fields = refdata.read_records(os.path.join(out, "fields.bin"))
    return info, fields


@pytest.mark.parametrize("name", ["cavity12_upwind", "warped5_corrected", "voronoi8_config2"])
def test_reference_program_with_b200_backend_converges_to_reference_fields(name):
    """Converges within 2 outer iterations of the reference's count; the fields after exactly the
    reference's count agree to 1e-8."""
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/babelsim-b200 is built only where the reference sources are present")
    g = Golden(name)
    target = int(g["conv_info"][1])
    info, fields = _run_program(g, 5000)
    assert abs(info["reported_iteration_intervals"] + 1 - target) <= 2
    if info["reported_iteration_intervals"] + 1 != target:
        info, fields = _run_program(g, target, never_converge=True)
    assert rel_l2(fields["U"].reshape(-1, 3), g["U_conv"]) < 1e-8
    assert rel_l2(fields["p"], g["p_conv"]) < 1e-8
