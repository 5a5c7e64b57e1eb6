"""CPU checkers for the DSMC engine.  TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and the CPU leg of bench.py may import
this package.  It holds:
  * the CPU restatement of the reference time step (dsmc_oracle.c), and
  * bindings to the reference's own routines compiled under the same stream
    contract (ref_shim/, built into _ref/ from the reference sources).
"""
