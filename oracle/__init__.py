"""ORACLE: test infrastructure for checking the B200 product path.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs may import this package, and only as the checker or the
timed CPU baseline -- never as the thing measured or shipped.

Contents
--------
* ``dense``  -- a numpy FP64 restatement of the reference's dense HOOI path
  (Function::ttm / gram / ttt_except, ALS_, HOOI_ALS).
* ``ref``    -- ctypes bindings to ``_ref/libdiana_ref.so``, the reference's
  own dense HOOI compiled in place from its sources (see ``Makefile``).
* ``sparse`` -- ctypes bindings to ``_build/libdt_oracle.so``, the plain-C
  restatement of the reference's sparse TTMc and sparse HOOI.

Pinning: ``tests/test_oracle.py`` checks the compiled reference and the
numpy restatement against the reference's own known-answer tests (TTM1,
Gram1) and against each other; the sparse restatement is pinned against the
compiled reference's dense ``Function::ttm`` chain on densified inputs.
"""
