"""Oracle package -- test infrastructure only (CPU restatement and reference pin).

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
arm.  Never imported by the heliocubed_b200 product package.
"""
