"""CPU oracle for the symmetric block-sparse hot path.

TEST INFRASTRUCTURE ONLY.  This package is a plain-Python/numpy restatement
of TeNeT's Host-path algorithms (sector codecs, fusion-tree enumeration,
coupled-sector block layout, F/R/B recoupling, per-sector composition,
blockwise SVD and truncation selection).  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it, and only as the checker or as the timed CPU baseline.  The product
(``tenet_b200``) never imports, links or executes anything in here.

Pinning: the restatement is checked against the golden vectors the reference
itself carries -- the TensorKit semantic oracle output
(``benchmarks/tensorkit_semantic_oracle.out``: SU(2)/fZ2/product symbol
tables, the U(1)/SU(2)/fZ2xU1xSU2 invariant streams, the planar repartition
fixtures and the weighted-rank truncation fixture) and the frozen SU(2)
values of ``tenet-sectors/src/su2.rs:377-470``.  Those fixtures are committed
under ``tests/golden/`` together with the script that extracted them.

Each function cites the reference file:line it follows (paths relative to
the TeNeT workspace root).
"""

from .sectors import Rule, U1, SU2, FZ2, Z2, product  # noqa: F401
from .fusion import Leg, HomSpace  # noqa: F401
from .tensor import TensorMap  # noqa: F401
