"""Oracle package (TEST INFRASTRUCTURE): CPU restatement of the MANS hot path.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this package. The product (``mans_b200``) never does.
"""
