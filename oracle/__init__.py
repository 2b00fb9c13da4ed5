"""ORACLE -- CPU restatement of dynamiqs' mesolve hot path.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference legs
of ``bench.py`` may import this package, and only as the checker (or as the timed CPU
baseline).  The product package ``dynamiqs_b200`` never imports it and has no CPU
fallback.

* ``rk``       -- Tsit5 / Dopri5 adaptive loop, initial step, controller, dense output
* ``lindblad`` -- Lindblad vector fields (hermitian / standard / vectorized) and the
                  sparse-DIA primitives
* ``mesolve``  -- one mesolve instance (saving, expects, infos)
* ``fp64``     -- independent FP64 references (scipy DOP853, Liouvillian expm)

Parity pins: see the module docstring of ``oracle.rk``.
"""
