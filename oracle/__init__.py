"""CPU oracle for the vlx-twoe-ints J/K path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The product (the package under
vlx-twoe-ints_b200/) never imports anything from here.
"""
