"""The host thread pool that stages pm_run's pageable operands, stressed on the CPU (no GPU).

A task set handed to the pool must run every task exactly once and have none still running
when the call returns: the tasks capture the caller's stack.  An earlier pool published a new
set's task count before closing the previous set's claim word, so a worker could claim a task
under the old set -- running it with a stale task pointer, or counting it into the new set so
that the call returned early; it crashed a pool's first call about once in a few thousand.
Both shapes are exercised: many fresh pools (a first call each) and long runs of task sets of
varying size."""
import pytest

from conftest import ensure_library


def test_first_calls_of_fresh_pools():
    import polymult
    ensure_library()
    assert polymult.host_pool_selftest(pools=3000, runs=2) == 0


def test_varying_task_counts():
    import polymult
    ensure_library()
    assert polymult.host_pool_selftest(pools=40, runs=1000, vary=True) == 0


def test_argument_check():
    import polymult
    ensure_library()
    with pytest.raises(polymult.PolymultError):
        polymult.host_pool_selftest(pools=1, runs=1, workers=100)
