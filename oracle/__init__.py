"""ORACLE -- test infrastructure only (CPU restatements of the reference's hot-path algorithms).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import this package, as the checker.
The product (``seq_vp_3d_b200``) never imports it.
"""
