"""The host thread pool that stages pm_run's pageable operands, stressed on the CPU (no GPU).

A task set handed to the pool must run every task exactly once and have none still running
when the call returns: the tasks capture the caller's stack.  The pool hands out tasks as
tickets of one packed word (job, count, next ticket) with fetch_add, and replaces the job's
function only after every task of the job has finished.  Four shapes are exercised: many fresh
pools (a first call each), long runs of task sets of varying size, task sets that find the
workers parked on their futex and must wake them, and task sets opened on the workers alone
(start) and joined by the caller after its own work (wait), as the staging pipeline does."""
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


def test_parked_workers_are_woken():
    import polymult
    ensure_library()
    assert polymult.host_pool_selftest(pools=4, runs=300, vary=True, park=True) == 0


def test_started_sets_joined_later():
    import polymult
    ensure_library()
    assert polymult.host_pool_selftest(pools=40, runs=1000, vary=True, split=True) == 0
    assert polymult.host_pool_selftest(pools=4, runs=300, vary=True, park=True, split=True) == 0
    # no workers: wait() runs every task on the caller
    assert polymult.host_pool_selftest(pools=20, runs=100, workers=0, vary=True, split=True) == 0


def test_argument_check():
    import polymult
    ensure_library()
    with pytest.raises(polymult.PolymultError):
        polymult.host_pool_selftest(pools=1, runs=1, workers=100)
