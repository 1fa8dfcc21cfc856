"""CPU FP64 oracle for the AIR Tools II SIRT/ART hot path.

TEST INFRASTRUCTURE ONLY.  This package restates the reference MATLAB code
(AIR Tools II V1.0, files cited per function) in NumPy/SciPy and in plain C.
It is the checker that the CUDA path is compared against.  Only the test
suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference arm of
``bench.py`` may import it; the product (``airtoolsii_b200``) never does.

Parity status: UNPINNED against MATLAB itself.  The reference ships no golden
vectors or tests, and neither MATLAB nor GNU Octave is installed, so the
reference .m files cannot be run here.  The restatement is instead pinned by
(i) the reference demos' invariants (matrix == pseudo-matrix-free ==
matrix-free operator, custom SIRT with empty struct == landweber, scaled
custom M == cimmino, constraints hold after every iteration), (ii) analytic
known answers of the ray tracer (axis-aligned rays, chord lengths), and
(iii) agreement of two independent restatements (NumPy and C) of the ray
tracer.
"""
