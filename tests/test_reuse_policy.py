"""Preconditioner lag (PcReusePolicy, babelsim_b200/csrc/linalg.h) against a restatement of the
reference's counters in PetscLinearSystem (src/backend/petsc_linear_system.cpp:257-324, 446-470).

The host struct is compiled with g++ into a small driver that replays a sequence of solves (matrix
changed or not, iterations, status) and prints, per solve, whether the preconditioner was rebuilt.
No GPU is needed.
"""
import os
import shutil
import subprocess

import pytest

from helpers import ReferenceCounters

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA_INCLUDE = "/usr/local/cuda/include"

DRIVER = r"""
#include "linalg.h"
#include <cstdio>
int main(int argc, char** argv) {
    bsg::PcReusePolicy p;
    bsg::SolverConfig c;
    c.rebuild_interval = 8;
    c.reuse_growth = 2.0;
    int changed, its, status;
    while (std::scanf("%d %d %d", &changed, &its, &status) == 3) {
        const bool rebuild = p.needRebuild(changed != 0, c);
        p.afterSolve(status, its, its, c);
        std::printf("%d\n", rebuild ? 1 : 0);
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INCLUDE):
        pytest.skip("needs g++ and the CUDA headers")
    d = tmp_path_factory.mktemp("reuse")
    src = d / "driver.cpp"
    src.write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["g++", "-std=c++17", f"-I{CUDA_INCLUDE}", f"-I{os.path.join(ROOT, 'babelsim_b200', 'csrc')}",
                    str(src), "-o", str(exe)], check=True)
    return exe


def _replay(exe, seq):
    out = subprocess.run([str(exe)], input="".join(f"{c} {i} {s}\n" for c, i, s in seq), capture_output=True,
                         text=True, check=True).stdout.split()
    return [o == "1" for o in out]


def _reference(seq, **kw):
    r = ReferenceCounters(**kw)
    return [r.solve(c, i, s) for c, i, s in seq]


def test_simple_schedule_three_solves_per_outer(driver):
    """SIMPLE: one new matrix per outer iteration, then two non-orthogonal corrector solves on it."""
    seq = [(1 if k % 3 == 0 else 0, 30, 0) for k in range(3 * 12)]
    mine = _replay(driver, seq)
    assert mine == _reference(seq)
    assert [k for k, r in enumerate(mine) if r] == [0, 9, 18, 27]   # rebuilt every third outer iteration


def test_one_solve_per_matrix_rebuilds_every_interval(driver):
    seq = [(1, 40, 0)] * 20
    mine = _replay(driver, seq)
    assert mine == _reference(seq)
    assert [k for k, r in enumerate(mine) if r] == [0, 8, 16]


def test_iteration_growth_forces_a_rebuild(driver):
    """A lagged solve needing more than twice the fresh iterations rebuilds before the next solve."""
    seq = [(1, 20, 0), (1, 25, 0), (1, 41, 0), (0, 20, 0), (1, 30, 0)]
    mine = _replay(driver, seq)
    assert mine == _reference(seq)
    assert mine == [True, False, False, True, False]
