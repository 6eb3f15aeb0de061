"""CPU oracle for the loki time-domain FFA / boxcar-score path.

Test infrastructure only. Two checkers live here:

* ``oracle.lko``: a ctypes binding of ``loki_oracle.c``, this project's plain-C
  restatement of the reference algorithm (built by ``make -C oracle oracle``).
* ``oracle.ref``: a ctypes binding of ``_ref/libloki_ref_*.so``, the
  reference's own CPU sources compiled unmodified (``make -C oracle ref``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
and reference legs may import this package. The product package
``loki_b200`` never imports it.
"""
