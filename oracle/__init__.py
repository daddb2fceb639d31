"""CPU oracle for the BabelSim SIMPLE hot path.  TEST INFRASTRUCTURE ONLY.

This package is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  It holds

* ``fvm``      - a numpy restatement of the reference's face-loop finite-volume
                 operators and LDU assembly (src/discretization/operators.cpp,
                 src/discretization/procedural_equation.cpp, include/babelsim/field.h);
* ``geometry`` - a restatement of Mesh::polyhedral geometry (src/core/mesh.cpp:321-564);
* ``simple``   - a restatement of the steady SIMPLE outer loop
                 (src/physics/simple/main.cpp:11-131) on top of ``fvm``;
* ``refdata``  - readers for the dumps written by the reference's own sources
                 compiled serially (``oracle/ref``, binary in ``oracle/_ref``).

Parity pinning: the restatement is checked against golden fixtures produced by
the reference's own finite-volume sources (tests/golden/make_golden.py), and
against the reference's analytic unit-test answers (tests/operators_test.cpp).
"""
