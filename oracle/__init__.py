"""CPU oracle for the IP pressure step -- test infrastructure.

Only `tests/`, `__graft_entry__.smoke()` and the CPU-baseline leg of
`bench.py` import this package, and only as the checker or the timed CPU
baseline.  The product (`implicitvelocityprojection_b200`) never imports it.
"""
