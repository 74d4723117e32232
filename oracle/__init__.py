"""CPU oracle for the B200 bundle adjuster -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may import this package.  It wraps oracle/_build/liboracle.so, a C++
restatement of RPBA's global LSA path (see rpba_oracle.cpp for the file:line
map).  Parity unpinned: the reference itself cannot be built here.
"""
from .oracle import *  # noqa: F401,F403
