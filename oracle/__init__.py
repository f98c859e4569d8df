"""Test oracle for the DVMpp hot path (CPU, FP64).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and
the cpu_baseline / reference legs of ``bench.py`` -- as the checker or as the
timed CPU baseline, never as the product.  ``dvmpp_b200`` does not import it.

Two oracles live here:

* ``port``: ``dvm_oracle.c`` -- a C restatement of the reference path, each
  function citing the reference lines it follows (``_ref/libdvmoracle.so``).
* ``ref``: the reference's own ``src/*.cpp`` compiled unmodified against a
  project-written Armadillo subset (``refshim/``) into ``_ref/libdvmref.so``
  by ``oracle/Makefile``.  It pins the port bit-for-bit.
"""
