"""CPU oracle for the TJM engine — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs may import
this package.  It restates the reference's algorithms in plain C++ FP64
(tjm_oracle.cpp) and numpy (dense.py) and is never part of the product.
"""
