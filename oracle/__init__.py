"""CPU oracle for the FSD velocity path -- TEST INFRASTRUCTURE ONLY.

Nothing in this package is part of the product: only the tests, the smoke
check in ``__graft_entry__`` and the CPU baseline leg of ``bench.py`` import
it, and only as the checker or the timed CPU restatement.

* ``oracle.fsd_oracle`` restates the reference's algorithm in NumPy (FP64):
  set-up, neighbour list, PSE mobility (spread / FFT / Green / contract and
  real space), lubrication pair products, saddle operator, preconditioner,
  GMRES.  Each function cites the reference file:line it follows.
* ``oracle.refbind`` loads ``oracle/_ref/libfsdref.so`` when it has been built
  (``python oracle/ref_recipe/build_ref.py``, needs the reference checkout):
  the reference's own per-thread device functions, set-up blocks and RCM,
  compiled for the host.  It pins the restatement; golden fixtures made from
  it are committed under ``tests/golden`` for machines without the checkout.
"""
