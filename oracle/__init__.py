"""CPU oracle for the fastLPR NUFFT path -- TEST INFRASTRUCTURE ONLY.

This package restates, in numpy/scipy, the reference fastLPR Python
algorithm for ``cv_fastlpr`` / ``cv_fastkde`` (reference package
``fastLPR_py/src/fastlpr``).  It is the checker for the CUDA path:

* ``tests/`` compare the GPU results against it,
* ``__graft_entry__.smoke()`` checks one small GPU call against it,
* ``bench.py`` times it as the CPU baseline (``cpu_baseline`` and
  ``--impl reference``).

Nothing in ``fastlpr_b200`` imports this package; the product path fails
loudly when its CUDA library is missing instead of falling back here.

Parity of this oracle is pinned by the golden fixtures in
``tests/golden/*.npz``, which ``tests/golden/make_golden.py`` produced by
running the reference itself (FP64 configuration) on seeded inputs.
"""
from .lpr import (  # noqa: F401
    cv_fastlpr,
    cv_fastkde,
    get_hlist,
    grid_params,
    knot_coordinates,
    spread_grid,
    nufft_spectra,
    kernel_spectra,
    design_powers,
    solve_system,
    linear_interp,
    one_se_rule,
    hutchinson_probes,
)
