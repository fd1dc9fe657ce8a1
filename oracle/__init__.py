"""CPU oracle for the Omniscape moving-window path (test infrastructure only).

Nothing in ``landschaft_b200`` imports this package.  It is loaded by the test
suite, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
``bench.py``, always as the checker or the timed CPU reference, never as the
product.
"""

from .oracle import (  # noqa: F401
    REF_AVAILABLE,
    advanced,
    core_omniscape,
    correction,
    count_targets,
    omniscape,
    omniscape_grad,
    port_lib,
    ref_advanced,
    ref_correction,
    ref_lib,
    source_from_resistance,
)
