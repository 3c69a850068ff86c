"""FP64 CPU oracle of the MSET hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference
leg may import this package.  The product (mset_b200/) never does.
"""
