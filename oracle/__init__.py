"""ORACLE -- test infrastructure only.

CPU restatement of the reference's numeric factorize / solve / refine path
(see oracle.hpp for the file:line map). Imported only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, as the checker.
"""
