"""CPU oracle for the QUDOS PWEM solve path -- TEST INFRASTRUCTURE ONLY.

This package is a plain numpy/scipy restatement of the reference algorithm
(QUDOS ``code/source/8_band``) used as the checker for the CUDA product in
``qudos_b200``.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` may import it.  The product path never calls it
and never falls back to it.

Every function cites the reference file and line range it follows.

Pinning: ``tests/test_oracle_golden.py`` checks the oracle end to end
against the reference's own golden outputs
(``code/example/Prism_111/Electronic_structure/PWEM_test_ref/energies_*.dat``),
which cover the closed-form shapes, anisotropic strain, first- and
second-order piezoelectricity, the identity strain-cell downsampling, the
assembly block map and the index-window eigensolve, plus the example's
Coulomb, momentum-matrix-element and probability-density outputs.  The lens
shape transform has no golden file in the reference; its integral ``I_J0`` is
evaluated the way the reference evaluates it, by GSL's adaptive 61-point
Gauss-Kronrod routine, restated in ``quadrature`` (GSL itself is an external
library that is not part of the checkout).
"""

from . import inputs, materials, shapes, strain, hamiltonian, eigen, coulomb, pipeline  # noqa: F401
