"""Test infrastructure: CPU oracle and reference-build drivers.

THIS PACKAGE IS NOT PART OF THE PRODUCT.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline / reference legs of
``bench.py`` may import it, and only as the checker or the baseline being
timed, never as the implementation under test.

* ``np_tomo``  - NumPy restatement (float32 "port" and float64 "accurate")
  of the reference's reconstruction path: dark/flat + -log
  (src/tomocupy/processing/proc_functions.py:55-83), filter spectrum and
  centred filtering (reconstruction/fbp_filter.py:60-118,
  reconstruction/backproj_functions.py:93-109), Fourier gridding
  (src/include/kernels_fourierrec.cuh, src/cuda/cfunc_fourierrec.cu:67-94)
  and line backprojection (src/include/kernels_linerec.cuh:3-137).
* ``refglue``  - drives the reference's own CUDA operators, compiled from
  the reference sources into ``oracle/_ref/`` by ``oracle/Makefile``, with a
  torch restatement of the reference's CuPy glue.  GPU only.

Parity pinning: the reference ships no golden vectors (its test fixtures
are absent).  The NumPy oracle is pinned against fixtures in
``tests/golden/`` that were produced by running the reference build
(``tests/golden/make_golden.py``) and, for the pure-Python parts (filter
spectrum, size bookkeeping), by executing the reference's Python source with
NumPy standing in for CuPy.
"""
