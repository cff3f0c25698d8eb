"""Oracle: CPU restatements of the reference algorithms (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package, and only as the checker / CPU baseline --
never as part of the product path.
"""
