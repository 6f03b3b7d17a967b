"""CPU oracle for the gradient-domain Poisson path (TEST INFRASTRUCTURE ONLY).

This package restates, in plain NumPy/SciPy, the algorithms of the reference
project ``gradient-domain`` (Giankaqui/visual-computing) for the Poisson
integration path: the discrete operators, the vertex-centred geometric
multigrid V-cycle, the four Dirichlet solvers, the DCT Neumann solver, the
masked (Perez) sparse solve and the tone-mapping attenuation.  Each function
cites the reference file and line range it follows.

It exists to check the CUDA implementation in ``gradient_domain_b200``.  Only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it, and only as the checker or the timed CPU baseline,
never as a code path of the product.

Parity pinning: ``tests/test_oracle.py`` checks this restatement against
golden vectors produced by the reference itself (``tests/golden/*.npz``,
generated by ``tests/golden/make_golden.py`` from the reference sources) and
against the known-answer assertions of the reference's own test suite.
"""

from . import hdr, multigrid, operators, poisson, solvers  # noqa: F401
