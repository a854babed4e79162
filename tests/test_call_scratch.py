"""CPU check of the per-call scratch of the device-pointer execute (fasttransforms_b200/csrc/api.cu,
execute_dev_impl / call_scratch): a call holds ntasks * (N / 16 + 2) progress words for the rotation
kernel's pass pipeline.  The pipeline needs one word per pass of every task, ceil(sweeps / wb) with
wb = 16, 32 or 64 sweeps a pass (the launch shapes' W x B); this restates the kernel's task list
and sweep counts (the formulas of tests/test_rot_staging.py) and checks that the words always
suffice, so the launcher's fallback (whole tasks per CTA when a queue needs more) never fires."""
import pytest

from test_rot_staging import DISK, SPH, TRI, default_M, task_sweeps, tasks


def words_needed(k, M, wb):
    return sum(-(-task_sweeps(k, M, mb, 0)[0] // wb) for mb in tasks(k, M))


@pytest.mark.parametrize("k", [SPH, TRI, DISK])
@pytest.mark.parametrize("n", [1, 2, 3, 16, 17, 63, 64, 65, 255, 256, 511, 1023, 1024, 2048, 4096])
def test_progress_words_suffice(k, n):
    for M in {default_M(k, n), max(1, default_M(k, n) // 3) | (0 if k == TRI else 1)}:
        if k == TRI and M != n:
            continue   # tri transforms take M == N only
        cap = len(tasks(k, M)) * (n // 16 + 2)
        for wb in (16, 32, 64):
            assert words_needed(k, M, wb) <= cap, (k, n, M, wb)


def test_sweeps_per_task_stay_below_n():
    # the bound above rests on a task having at most n sweeps
    for k in (SPH, TRI, DISK):
        for n in (5, 64, 300, 1024):
            M = default_M(k, n)
            assert max((task_sweeps(k, M, mb, 0)[0] for mb in tasks(k, M)), default=0) <= n
