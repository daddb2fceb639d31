"""The allocation-free PCG entry point (bsg_pcg_jacobi_static) against bsg_solve_ldu.

bsg_pcg_jacobi_static keeps its scratch in a static device array inside the
library; it is for callers that cannot allocate device memory while running.
This file is collected last so that it also runs after every other test in the
same process.  Tolerance: relative L2 1e-8, the tolerance the linear-solve
parity tests use (rtol 1e-12 solves).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import Golden, ref_system_groups, rel_l2
from oracle import fvm

pytestmark = pytest.mark.gpu


def test_static_pcg_matches_solve_ldu():
    import scipy.sparse as sp
    import torch
    import babelsim_b200 as bsg
    from babelsim_b200 import _lib

    g = Golden("cavity64_config1")
    sysp = ref_system_groups(g)[0]["pressure"][0]
    ldu = fvm.LDU(g.oracle_geometry(), False)
    ldu.diag, ldu.upper, ldu.lower, ldu.source = sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"]
    full = sp.csr_matrix(ldu.matrix())
    n = full.shape[0]
    off = sp.csr_matrix(full - sp.diags(full.diagonal()))
    off.eliminate_zeros()
    off.sort_indices()

    # the existing entry point: CG + Jacobi through the mesh-bound LDU solve
    ctx = bsg.Context(0)
    try:
        mesh = bsg.Mesh.from_polyhedral(ctx, g.poly)
        cfg = bsg.solver_config("cg", "jacobi", 1e-30, 1e-12, 20000)
        x_ref, res_ref = bsg.solve_ldu(mesh, cfg, sysp["diag"], sysp["upper"], sysp["lower"], sysp["source"])
        assert res_ref[0].status == 0

        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        row_ptr = torch.tensor(off.indptr.astype(np.int32), device=dev)
        cols = torch.tensor(off.indices.astype(np.int32), device=dev)
        vals = torch.tensor(off.data.astype(np.float64), device=dev)
        diag = torch.tensor(np.ascontiguousarray(full.diagonal(), np.float64), device=dev)
        b = torch.tensor(np.ascontiguousarray(sysp["source"], np.float64), device=dev)
        torch.cuda.synchronize()

        L = _lib.lib()
        results = []
        for _ in range(2):
            x = torch.full((n,), 7.0, dtype=torch.float64, device=dev)   # overwritten: zero initial guess
            res = _lib.SolveResult()
            _lib.check(L.bsg_pcg_jacobi_static(n, C.c_void_p(row_ptr.data_ptr()), C.c_void_p(cols.data_ptr()),
                                               C.c_void_p(diag.data_ptr()), C.c_void_p(vals.data_ptr()),
                                               C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1e-30, 1e-12,
                                               20000, C.byref(res)))
            assert res.status == 0
            assert res.final_residual <= 1e-12 * np.linalg.norm(sysp["source"]) * 1.0000001
            results.append(x.cpu().numpy())
        for x in results:
            assert rel_l2(x, x_ref) < 1e-8
        assert rel_l2(results[0], results[1]) < 1e-8

        # sizes beyond the static scratch are rejected before any device work
        res = _lib.SolveResult()
        code = L.bsg_pcg_jacobi_static(131073, None, None, None, None, None, None, 1e-30, 1e-12, 10, C.byref(res))
        assert code == 1   # BSG_ERR_ARGUMENT
        assert b"131072" in L.bsg_global_error()
    finally:
        ctx.close()
