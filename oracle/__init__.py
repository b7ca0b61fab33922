"""CPU oracle for the Sinkhorn hot path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this package, and only as the checker.  The product package
``ott_b200`` never imports it.
"""
