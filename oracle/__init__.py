"""CPU oracle for the pseudo-spectral Taylor-Green RK3 step (test infrastructure only).

Nothing in ``spectral_solver_b200`` imports this package.  It is used by ``tests/`` as the
checker, by ``__graft_entry__.smoke()`` as the checker, and by ``bench.py`` as the timed
CPU baseline (``cpu_baseline`` and ``--impl reference``).  Every function cites the
file:line of ovankerm/Spectral_solver that it restates.
"""
