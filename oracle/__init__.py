"""CPU oracle for the ms2dirty / dirty2ms hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this package, and only as the checker; the product (curig_b200) never imports
it and has no CPU fallback.
"""
