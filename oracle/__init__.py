"""CPU oracle for the twist-mesh pipeline -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's double-precision CPU path (rlm_cpu_dp and
hlm_cpu_dp of qiongz/Random-Landau-Model); every function cites the reference
file:line it follows.  It is the checker for the CUDA product: only the tests,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arms may
import it, and never as the thing measured or shipped.

Pinning: ``oracle/Makefile`` compiles the reference's own sources (with the MKL shim
in ``oracle/shim``) into ``oracle/_ref``; ``tests/golden/make_golden.py`` records
their full-precision outputs as fixtures, and ``tests/test_oracle_golden.py`` checks
this restatement against those fixtures.
"""
