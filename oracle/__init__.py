"""CPU oracle for the alignment hot path -- test infrastructure only.

Imported by the test suite, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` as the parity checker; the shipped library never uses it.
"""
