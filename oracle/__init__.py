"""Test infrastructure: the CPU oracle (restatement of the reference) and the reference
build. Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg."""
