"""CPU oracle of the sphere-tracing pass: TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
as the checker; the product path never imports it.
"""
