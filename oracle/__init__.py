"""Oracle package: the CPU checker for the B200 transform path.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() and
by bench.py's cpu_baseline / reference legs -- never by the product package
(fastandfourier_b200), which must fail loudly rather than fall back to CPU.

  oracle.orc      -- ctypes bindings to liboracle.so, the C restatement of the
                     reference algorithms (faf_oracle.c), plus FP64 numpy DFTs.
  oracle.refimpl  -- ctypes bindings to the reference library itself, compiled
                     from its own sources by oracle/Makefile into oracle/_ref/.
"""
