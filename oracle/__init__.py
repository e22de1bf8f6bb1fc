"""CPU oracle for the FDFD solve path (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import this package, and only as the checker or the timed CPU
baseline.  The product package (``meanas_b200``) never imports it.
"""
