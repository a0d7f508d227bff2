"""CPU oracle for the standard-gridder imaging path (TEST INFRASTRUCTURE).

This package restates astroviper's CPU arithmetic for the hot path so that the
CUDA kernels of ``astroviper_b200`` can be checked against it:

* ``av_oracle.c`` (built into ``liboracle.so`` by ``build.sh``): the FP64
  gridder (``standard_grid_jit``, standard_grid.py:246-432), degridder
  (``dgrid_numba``, standard_degrid.py:388-485), imaging-weight grid/degrid
  (grid_imaging_weights.py:93-206, :285-443), the PSWF functions
  (gcf_prolate_spheroidal.py:87-158) and Hogbom CLEAN (hclean.cpp:51-210),
  in the reference's operation order;
* numpy restatements of the grid-correction + FFT image formation
  (standard_grid.py:693-708), the FFT helpers (fft.py:5, ifft.py:5) and the
  Briggs factors (briggs_weighting.py:1-31).

Parity of this oracle with the reference itself is pinned by
``tests/golden`` (fixtures generated from the reference's own Numba and C++
code by ``tests/golden/make_golden.py``) and checked by
``tests/test_oracle_golden.py``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package; the product never does.
"""
from .oracle import *  # noqa: F401,F403
