"""TEST INFRASTRUCTURE ONLY — the CPU oracle and the reference-kernel harness.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU legs, never by
the product package.
"""
