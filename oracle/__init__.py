"""ORACLE: CPU restatements of the reference's algorithms, used only as the
checker by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.
Nothing in the product package imports this package."""
