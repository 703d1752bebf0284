"""TEST INFRASTRUCTURE ONLY: the oracle (CPU restatement) and the reference build.

Imported only by tests/, __graft_entry__.smoke() and bench.py's baseline legs,
always as the checker or the timed baseline, never as the product.
"""
