"""TEST ORACLE ONLY -- the checker for the snuqs_b200 engine.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only to check results or to time the
reference CPU path.  The product (``snuqs_b200``) never imports it.

Two oracles live here:

* ``liboracle.so`` (``sq_oracle.c``): a plain-C restatement of the reference's
  CPU gate path (``gate_operations_impl_cpu.cc:10-148``) and gate matrices
  (``gate_operations.cc:9-734``).
* ``_ref/libsnuqs_ref.so``: the reference's own CPU gate path compiled from its
  sources (``oracle/Makefile``).  It pins the restatement bit for bit.

Plus numpy restatements of what the reference lacks (Pauli-string
expectation, probabilities, sampling helpers) and of its gate reordering
(``transpile.py:33-89``).
"""
from .oracle import *  # noqa: F401,F403
