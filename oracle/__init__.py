"""CPU oracle for the ChainAMPS DMRG hot path.

Test infrastructure only: a numpy restatement of the reference's algorithm,
used as the checker for the CUDA library by ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``.  The product
path never imports it.  Each function cites the reference file:line it
follows.  Pinned against the reference's example outputs
(``tests/golden/kat_examples.json``).
"""
