"""Test infrastructure: CPU restatements of OpenKSpace's ``cs`` path.

Nothing in this package is product code.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it, and only as the checker (or the timed CPU baseline), never as the thing
that is measured or shipped.

* ``cs_fp64``  -- numpy complex128 restatement (the FP64 oracle).
* ``cs_ref.c`` -- FP32 C restatement that follows the reference's operation
  order (built into ``oracle/_ref/libcsref.so`` by ``oracle/Makefile``); the
  stand-in for the reference ``cs`` output and the timed CPU baseline.
* ``csref``    -- ctypes wrapper around ``libcsref.so``.

Parity pins: both restatements are checked against every known-answer and
property test the reference holds for this path (restated in
``tests/test_oracle_pins.py``).  Bit-level parity with ``rustfft`` 6.4.1 is
unpinned (the reference ships no golden vectors and cannot be built here);
the 1e-4 relative-L2 tolerance covers any accurate FFT.
"""
