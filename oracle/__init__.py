"""CPU oracle for parity tests (test infrastructure, never the product path).

Importable only from tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg.
"""
