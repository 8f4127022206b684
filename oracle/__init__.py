"""CPU oracle of the palette-weight rasterizer -- TEST INFRASTRUCTURE ONLY.

A from-scratch restatement of the reference gsplatcu arithmetic (FP32 and
FP64) used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
as the checker.  The product (reparamgs-palette_b200/) never imports it.
"""
