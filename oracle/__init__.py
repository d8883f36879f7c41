"""CPU restatement of the cdft hot path, used ONLY as a checker.

This package is test infrastructure. It restates, in numpy (and scipy.sparse for the two
interpolation operators), the algorithms of the reference solver ``cdft`` for the path the CUDA
library replaces: the cusp-factorised staggered-divergence Hamiltonian apply, the Chebyshev-filtered
subspace iteration with its Rayleigh--Ritz step, the Coulomb-cutoff FFT Poisson solve, the VWN-LDA
and PBE exchange--correlation evaluation with the cusp-aware quadrature, and the SCF driver around
them. Every function cites the reference file and line it follows (paths are inside the reference
project, e.g. ``src/cdft/operators/divergence.py:172``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg (and its
``--impl reference`` arm) may import this package, and only to check or to time the CPU path. The
product package never imports it.

Parity pin: ``tests/golden/`` holds fixtures produced by running the reference itself in the build
container (``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py`` checks this package
against them and against the reference's own golden values (``tests/golden/values.json`` of the
reference, re-stated in the fixture file).

Random starts use torch's CPU generator, exactly as the reference's ``seeded_randn``
(``src/cdft/precision.py:246``) does, so that a seeded solve here draws the same numbers.
"""
