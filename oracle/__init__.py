"""CPU checkers for the traced path - TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package. It never serves a product call.
"""
