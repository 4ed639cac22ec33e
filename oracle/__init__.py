"""TEST INFRASTRUCTURE ONLY: the CPU oracle for the Sinkhorn WMD solve.

Imported by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py, and by nothing else.  Two checkers live here:

* ``liboracle.so`` (``wmd_oracle.c``): an FP64 restatement of the reference's
  fused solver ``sinkhorn_wmd_fused.cpp:112-393`` plus a converged mode and the
  stable counting-sort CSR/CSC builders (``sinkhorn_wmd_fused.cpp:493-506``).
* ``_ref/libref_{fused,nonfused}.so``: the reference's own ``sinkhorn_wmd``
  compiled from its sources in place by ``oracle/Makefile`` (present only where
  the reference checkout was available at build time).
"""
from .oracle import (  # noqa: F401
    OracleUnavailable,
    csc_from_csr,
    csr_from_csc,
    counting_sort,
    oracle_lib_path,
    reference_available,
    reference_sinkhorn,
    sinkhorn,
    sinkhorn_converged,
    select,
)
