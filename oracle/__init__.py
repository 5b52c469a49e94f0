"""Test infrastructure: CPU oracles for the ms3 bandpass_filter + whiten path.

Only tests/, __graft_entry__.smoke() and bench.py (CPU baseline and the
reference arm) may import this package.  The product library never does.
"""
