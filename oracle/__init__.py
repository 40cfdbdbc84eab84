"""CPU oracle for the ARW integration step (TEST INFRASTRUCTURE ONLY).

A numpy restatement of the reference's algorithm for the RK3 step
(pywrf/solver.py:709-1910 and the kernel modules it calls).  Every function
cites the reference lines it follows and writes exactly the index regions the
reference writes, so that halos and persistent work buffers evolve the same
way across steps.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or the timed
CPU baseline.  The product path (``pywrf_b200``) never imports it and fails
loudly when its CUDA library is missing.

Parity pin: the oracle is checked against golden fixtures produced by running
the reference itself (tests/golden/make_golden.py) in tests/test_oracle.py.
"""
from .model import OracleModel  # noqa: F401
