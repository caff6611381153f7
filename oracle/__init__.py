"""CPU oracle for the nodal-DG hot path: test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference arm
use this package, always as the checker (or the timed CPU restatement of the
reference), never as part of the product path.
"""
