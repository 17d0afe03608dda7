"""CPU oracle of the SAP contact step -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg and
reference arm may import this package, and only as the checker.  The product
(sap_warp_b200) never imports it.  Parity status: partially pinned (analytic
known-answer cases; no reference-run vectors exist because the reference
requires NVIDIA Warp, which is not importable here).
"""
