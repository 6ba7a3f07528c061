"""Test infrastructure only: the CPU oracles of the hot path.

* ``O2`` -- oracle/o2f_oracle.c, a sequential FP64 C restatement of the
  reference algorithm, loaded through ctypes (oracle.cpu).
* ``O1`` -- the reference solver's own sources compiled by
  oracle/build_ref.sh into oracle/_ref/ and driven as a subprocess
  (oracle.ref).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
use this package, always as the checker; the product never imports it.
"""
