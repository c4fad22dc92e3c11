"""The CPU oracle (test infrastructure): a restatement of vyges-gpl's global_placement path.

Only the tests, `__graft_entry__.smoke()` and `bench.py`'s CPU-baseline leg load it, as the
checker; the engine never does.
"""
from .oracle_py import Session, build, global_placement, lib  # noqa: F401
