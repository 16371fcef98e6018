"""CPU oracle for the cross-correlation PIV hot path (TEST INFRASTRUCTURE ONLY).

This package restates, in NumPy Float64 and plain C++, the per-interrogation-area
algorithm of Marc-3d/multi_quickPIV (Julia).  It exists to check the CUDA
product path; the product never imports it.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import or run anything in here.

Parity status: the reference's own test suite is empty (``test/runtests.jl``
and ``test/fft_r2c_tests.jl`` are 0 bytes) and Julia/FFTW are absent on this
machine, so no reference output pins this restatement ("parity unpinned" at
the FFTW boundary).  It is instead pinned by (1) brute-force spatial
correlation, (2) integer-shift and sub-pixel known-answer tests, and (3) unit
tests of every reference quirk the path depends on; the fixtures it produced
are committed under ``tests/golden/``.
"""
