"""CPU oracle for cellweave's hot path: test infrastructure only.

A C restatement of the reference's Rust functions (``cw_oracle.c``) with a
ctypes face (``oracle.py``).  Only the tests, the smoke check and the
benchmark's CPU-baseline leg use it, as the checker; no product code path
imports it.
"""
