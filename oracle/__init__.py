"""CPU oracle for the SpGEMM engine -- test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker.  See spgemm_oracle.c for what it
restates from the reference.
"""
