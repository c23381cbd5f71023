"""CPU oracle of the jax-fli particle-mesh path — TEST INFRASTRUCTURE ONLY.

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, as
the checker. The product package (jfli_b200) never imports anything from here.
"""
