"""CPU FP64 oracle for the periodicflow right-hand-side and time-stepping path.

TEST INFRASTRUCTURE ONLY.  This package is the checker, never the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it.  The product package
(``periodic-flow_b200/periodicflow``) never imports, links or calls anything here.
"""
from .pf_oracle import *  # noqa: F401,F403
