"""ORACLE — test infrastructure only.

CPU restatements used by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline as the checker; nothing in ordinarylight_b200/ imports this package.
"""
