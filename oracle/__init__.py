"""Test infrastructure: the CPU oracle (oracle.cpp) and the harness around the
reference's own kernels (ref/). Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg use this package; the product never does."""
