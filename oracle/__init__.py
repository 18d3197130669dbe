"""ORACLE: CPU restatements of the reference's hot path, used only as the checker.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this package. The
product (nabladyn_b200) never does.
"""
