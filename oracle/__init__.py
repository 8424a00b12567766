"""CPU oracle for the SpGEMM engine -- test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this package, and only as the checker.  See spgemm_oracle.c for what it
restates from the reference.
"""

import os as _os


def reference_root():
    """Directory of the reference sources, or None when they are absent:
    $RTSPMSPM_REFERENCE, else a directory named ``reference`` beside the
    repository."""
    cand = _os.environ.get("RTSPMSPM_REFERENCE") or _os.path.join(
        _os.path.dirname(_os.path.dirname(_os.path.dirname(_os.path.abspath(__file__)))), "reference")
    return cand if _os.path.isdir(cand) else None
