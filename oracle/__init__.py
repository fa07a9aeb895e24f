"""CPU oracle for the static-exchange per-energy scattering path.

TEST INFRASTRUCTURE ONLY.  This package is a plain numpy/scipy restatement
of the reference C++ hot path (SchurInverter -> ForwardRPropagator ->
KMatrixExtractor -> BackPropagator -> AsymptoticAmplitudes ->
DipoleMatrixElement) used as the checker for the CUDA library.  Only the
test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it.  The product path never calls into it and
fails loudly when the CUDA extension is missing.

Each function cites the reference file:line it restates (paths relative to
the reference project root).  Dense linear algebra goes through the same
LAPACK routines the reference's MKL build calls (dgetrf/dgetri for the
general inverse, dsytrf/dsytri on the LOWER triangle for the Schur
inverse), here via scipy's bundled OpenBLAS.

Parity pinning: the angular algebra (3j / Gaunt / real-Y dipole table),
Simpson quadrature and the free-particle dipole are pinned to the golden
vectors of the reference's own unit tests (tests/golden/); the Riccati
functions are pinned to mpmath.  The end-to-end K / A / B / dipole values
cannot be pinned to the reference binary (it needs Eigen, HDF5 and GSL,
none of which exist in this image), so the end-to-end restatement is
"parity unpinned" against the reference binary.  It is checked instead
against the acceptance criteria of the reference's component tests, with
their thresholds (tests/test_oracle_properties.py, tests/test_oracle_blocks.py,
tests/test_oracle_gauge.py, tests/test_oracle_potential.py,
tests/test_oracle_gaunt_l50.py): the W^-1 operator against an LU inverse of the
assembled W, Sinv S = I, the exchange coupling against the triple loop, the
analytic start and an independent LU recursion, the three-point Numerov
identity on the back-propagated solution, K symmetry, S unitarity,
eigenphases, matching-radius invariance, the asymptotic-fit checks, the
setup rules, the per-channel length/velocity gauge identity, the channel
potential and the real Gaunt coefficients to l = 50.  K is also held to
exact phase shifts of a short-range well (tests/test_oracle_phase_shifts.py).

oracle/adjoint.py is the gradient checker for the adjoint (the reference
has none): the forward path restated in float64 torch and differentiated by
reverse mode, held to central finite differences of this oracle
(tests/test_adjoint_oracle.py).
"""
