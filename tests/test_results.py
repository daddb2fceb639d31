"""Result output in the reference's format: the reference's own restart reader loads what
bsg_write_results wrote, bit for bit (host only; runs the reference build in oracle/_ref)."""
import os
import sys

import numpy as np
import pytest

from helpers import ROOT, Golden

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
ORACLE = os.path.join(ROOT, "oracle", "_ref", "babelsim-oracle")


def test_written_files_have_the_reference_layout(tmp_path):
    import babelsim_b200 as bsg
    g = Golden("warped5_corrected")
    U, p = g["U_3"], g["p_3"]
    out = tmp_path / "final"
    bsg.write_results(out, "final", g.poly, {"U": U, "p": p})
    rank = out / "rank-0000"
    meta = (rank / "metadata.bs").read_text().splitlines()
    assert meta[:6] == ["format babelsim_result 3", "time final", "rank 0", "ranks 1",
                        f"global_cell_count {len(p)}", f"owned_cells {len(p)}"]
    assert "field U vector cell" in meta and "field p scalar cell" in meta
    rows = (rank / "U.csv").read_text().splitlines()
    assert rows[0] == "global_id,x,y,z,value0,value1,value2" and len(rows) == len(p) + 1
    vals = np.array([[float(v) for v in r.split(",")[4:]] for r in rows[1:]])
    assert np.array_equal(vals, U)  # 17 significant digits round-trip exactly
    geo = (rank / "mesh.geometry").read_text().splitlines()
    assert len(geo) == len(p) and geo[0].split(",")[1] == "8"  # hexahedra: 8 sorted unique vertices


@pytest.mark.skipif(not os.path.exists(ORACLE), reason="reference build (oracle/_ref) not present")
def test_reference_restarts_from_written_results(tmp_path):
    """The reference's SIMPLE restarted from our result files computes exactly what it computes
    from the same values given as its own nonuniform data files."""
    import babelsim_b200 as bsg
    from make_golden import config1_solution, methods, run, write_case
    g = Golden("cavity12_upwind")
    U, p = g["U_3"], g["p_3"]
    res = tmp_path / "results" / "final"
    bsg.write_results(res, "final", g.poly, {"U": U, "p": p})
    m = g.meta
    U_bcs = [(t, tuple(v)) for t, v in m["U_bcs"]]
    p_bcs = [(t, v) for t, v in m["p_bcs"]]
    physics = {"density": 1.0, "dynamicViscosity": 0.01}
    a = tmp_path / "restart"
    write_case(str(a), g.poly, U_bcs, p_bcs, methods(), config1_solution(1e-12), physics,
               internal={"U": f"file {res}", "p": f"file {res}"})
    b = tmp_path / "datafiles"
    write_case(str(b), g.poly, U_bcs, p_bcs, methods(), config1_solution(1e-12), physics,
               internal={"U": "file U.dat", "p": "file p.dat"})
    with open(b / "fields" / "initial" / "U.dat", "w") as f:
        f.writelines(f"{i} {float(u[0])!r} {float(u[1])!r} {float(u[2])!r}\n" for i, u in enumerate(U))
    with open(b / "fields" / "initial" / "p.dat", "w") as f:
        f.writelines(f"{i} {float(v)!r}\n" for i, v in enumerate(p))
    fa, _, ia, _ = run(str(a), 1)
    fb, _, ib, _ = run(str(b), 1)
    for key in ("U", "p", "phi"):
        assert np.array_equal(fa[key], fb[key]), key
    assert not np.array_equal(fa["U"].reshape(-1, 3), U)  # one more iteration did happen
