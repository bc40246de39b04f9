"""TEST INFRASTRUCTURE ONLY -- the CPU oracle (checker).

Importable only by tests/, bench.py's CPU-baseline leg and
__graft_entry__.smoke(); the product (spectral_upcxx_b200) never imports it.
"""
