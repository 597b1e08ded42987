"""CPU oracle for the B200 step loop: test infrastructure, never the product.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package.
"""
