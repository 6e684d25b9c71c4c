"""CPU oracle for the Swendsen-Wang sweep (test infrastructure only).

Only the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package.  It restates the reference algorithm of
Amirhossein-Manouchehri/rbim-fk-percolation in plain C (``rbim_oracle.c``) and
Python (``winding.py``), with numpy's PCG64 draws replaced by the Philox4x32-10
stream of the CUDA engine so that chains can be replayed bit for bit.

Parity of the restatement is pinned by ``tests/test_oracle_golden.py`` against
golden vectors that ``tests/golden/make_golden.py`` produced by running the
reference itself.
"""

from .oracle import *  # noqa: F401,F403
from .oracle import __all__ as _oracle_all
from .winding import spanning_forest_winding  # noqa: F401

__all__ = list(_oracle_all) + ["spanning_forest_winding"]
