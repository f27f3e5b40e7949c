"""The oracle: test infrastructure that states what the reference computes.

Two independent sources, both CPU-only:

* ``oracle.port`` -- the project's C++ restatement of the reference's
  MPI-layer Bine collectives (oracle/bine_oracle.cc), loaded with ctypes.
* ``oracle.ref`` -- the unmodified reference library itself, compiled from
  its own sources against the project's MPI shim (oracle/Makefile ``ref``)
  and run as one forked process per rank (oracle/_ref/bine_ref_run).

Only tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package; the product never does.
"""
