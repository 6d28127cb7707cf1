"""CPU oracle for the par2-rs erasure-coding path -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of bench.py may import this package, and only as the
parity reference the GPU results are compared with or as the timed CPU
baseline.  The CUDA product never calls it.
"""
