"""Parity checker (TEST INFRASTRUCTURE ONLY).

``oracle/fdtd_oracle.c`` is a CPU restatement of the reference's FDTD path;
``oracle/_ref/deepgpr_cpu.so`` is the reference's own C/OpenMP backend
compiled from its source.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg use this package; the product never does.
"""
