"""Checkers for the GPU halo finder -- TEST INFRASTRUCTURE ONLY.

``oracle.cpu`` wraps the CPU restatement (fof_oracle.c) and
``oracle.reference`` drives the reference's own binaries built by
oracle/Makefile into oracle/_ref.  Only tests/, the smoke check and bench.py's
CPU-baseline / reference legs may use this package; the product path never
does.
"""
