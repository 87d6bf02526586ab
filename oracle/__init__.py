"""Test infrastructure: CPU checkers of the SIMPLE hot path.

Only tests/, __graft_entry__.smoke() and the CPU-baseline leg of bench.py
may import this package.  It never backs a product code path.
"""
