"""ORACLE -- test infrastructure only.

CPU restatements of the reference's hot path, used by tests/, by
``__graft_entry__.smoke()`` and by ``bench.py``'s CPU-baseline leg as the
checker.  The product package ``ccsd_gpu_b200`` never imports this package.
"""
