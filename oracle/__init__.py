"""CPU oracle (test infrastructure only; never imported by the product).

See ``oracle/dense_sht.py`` for what it restates and how it is pinned.
"""
