"""Test infrastructure: the CPU restatement of the reference (oracle.py) and
the reference's own CUDA kernels compiled from source (reference.py).  Only
tests/, __graft_entry__.smoke() and bench.py's baseline legs use this package."""
