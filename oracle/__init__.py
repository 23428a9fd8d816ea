"""CPU oracle for the batched flux-balance LP path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product package imports this directory.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference legs
use it, and only to check results (or as the timed CPU reference), never as a
solver behind the product API.

Contents
--------
``highs``        HiGHS through ``scipy.optimize.linprog`` (the reference's exact
                 CPU LP call, ``src/dfba_simulator.py:1081-1091`` and the
                 ``ParallelCpuLP`` thread-pool pattern of
                 ``scripts/microbatch_comparison_support.py:12-30``).  HiGHS is
                 a third-party dependency of the reference (``requirements.txt:4``
                 pins ``highspy>=1.15.1``); here it is the HiGHS 1.12.0 bundled
                 with SciPy 1.18.1.
``certificate``  restatement of the reference's original-LP certificate
                 (``src/cpu_repeated_lp.py:150-178``,
                 ``src/gpu_block_lp.py:52-132``).
``reference_pdhg`` restatement of the reference's plain FP64 PDHG operator and
                 Pock-Chambolle metric (``src/gpu_pdhg_corrector.py:183-200,
                 334-358``; ``tests/test_gpu_pdhg_workspace.py:35-50``).
``pdhg``         NumPy restatement of this engine's restarted Halpern PDHG
                 (preprocessing, iteration, restart rule, primal-weight update,
                 FP64 convergence test) -- the parity reference for the CUDA
                 kernels.
``dfba``         restatement of the dFBA coupling (Michaelis-Menten uptake
                 bounds, Euler biomass / medium update) from
                 ``src/dfba_simulator.py``.

Pinning: ``tests/test_oracle_pins.py`` checks these restatements against the
reference's own known-answer tests and against golden vectors produced by
importing the reference's ``_problem`` / ``_certificate`` (see
``tests/golden/make_golden.py``), and against HiGHS optima.
"""
