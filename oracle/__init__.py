"""CPU oracle: a numpy restatement of gridfoam's per-iteration hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in ``gridfoam_b200`` imports this
package; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, and only as the checker (or as the timed CPU
baseline), never as the product path.

Every function restates the float64 PyTorch algorithm of the reference
gridfoam v0.3.0 and cites the reference file and lines it follows (paths
relative to ``src/gridfoam``).  The restatement is pinned against golden
vectors produced by running the reference itself (``tests/golden``,
generated by ``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py``
checks that pin.
"""

from oracle.algorithms import PIMPLE, PISO, SIMPLE, create_algorithm
from oracle.case import Case

__all__ = ["Case", "SIMPLE", "PISO", "PIMPLE", "create_algorithm"]
