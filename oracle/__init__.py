"""CPU oracle for the orbital-evaluation path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this package, and only as the checker.  The product library never loads it.
"""
