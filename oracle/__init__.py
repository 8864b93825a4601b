"""TEST INFRASTRUCTURE -- the CPU oracle for the BIT treecode hot path.

Only tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and the
``--impl reference`` arm) import this package, and only as the checker or the timed CPU
baseline.  Nothing in ``bit_b200`` imports it.

``oracle.orc``  -- this project's C restatement (oracle/bit_oracle.c, built to lib/liborc.so)
``oracle.ref``  -- the unmodified reference treecode built from its own sources
                   (oracle/ref_wrap.cpp, built to _ref/libref_<tag>.so), when present.
"""
