"""CPU restatement of the rotation kernel's pass-pipeline queue (fasttransforms_b200/csrc/rotations.cu,
schedule_passes) on the kernel's task geometry (the formulas of tests/test_rot_staging.py).

A queue entry (task, prog0, first, stride) runs passes first, first + stride, ... of its task;
pass r > 0 of a pipelined entry waits for the progress word prog0 + r - 1 of the same task.
Checked for every family, several sizes, the launch shapes' pass lengths (16, 32, 64 sweeps),
all sweeps and heads-only lists, and both queue modes:
  * every pass of every task runs exactly once;
  * each task's progress words are its own (prog0 .. prog0 + passes - 1, disjoint, nprog in all);
  * a pipelined pass is queued after its task's previous pass, so the CTA it waits for pulled
    its entry earlier and is running (the queue cannot deadlock with one resident wave);
  * mode 2 pipelines only a prefix of the list (the longest tasks) and runs the rest whole."""
import pytest

from test_rot_staging import DISK, RECT, SPH, SPIN, TRI, default_M, task_orders, task_sweeps, tasks

L2 = 126 * 1024 * 1024     # B200 L2 bytes (cudaDevAttrL2CacheSize)


def schedule(k, N, M, wb, mode, blk=0):
    """The queue and progress-word count schedule_passes builds for the task list of (k, M)."""
    tl = tasks(k, M)
    npass = [-(-task_sweeps(k, M, mb, blk)[0] // wb) for mb in tl]
    prog0, nprog = [], 0
    for p in npass:
        prog0.append(nprog)
        nprog += p
    nt = len(tl)
    npipe = nt
    if mode == 2:
        seqs = 1 if k in (TRI, RECT) else (4 if k == SPIN else 2)   # doubles per order and row
        foot = task_orders(k) * seqs * N * 8
        npipe = min(nt, max(1, (L2 // 2) // max(foot, 1)))
    q = []
    for r in range(max(npass, default=0)):
        for t in range(npipe):
            if r < npass[t]:
                q.append((t, prog0[t], r, npass[t]))
    for t in range(npipe, nt):
        if npass[t] > 0:
            q.append((t, prog0[t], 0, 1))
    return q, npass, nprog, npipe


@pytest.mark.parametrize("k", [SPH, TRI, DISK])
@pytest.mark.parametrize("n", [17, 64, 255, 1024, 4096])
@pytest.mark.parametrize("wb", [16, 32, 64])
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("blk", [0, 32])
def test_pass_queue(k, n, wb, mode, blk):
    M = default_M(k, n)
    q, npass, nprog, npipe = schedule(k, n, M, wb, mode, blk)
    ran = {}
    pos = {}
    for i, (t, p0, first, stride) in enumerate(q):
        assert stride >= 1 and 0 <= first < npass[t]
        for r in range(first, npass[t], stride):
            assert (t, r) not in ran, (t, r)
            ran[(t, r)] = i
        pos.setdefault(t, []).append(i)
        if stride == npass[t] and first > 0:          # a pipelined pass waits for its predecessor
            assert ran[(t, first - 1)] < i
    assert sorted(ran) == sorted((t, r) for t in range(len(npass)) for r in range(npass[t]))
    # progress words: task t owns prog0 .. prog0 + npass - 1, all disjoint
    words = set()
    for t, p0, first, stride in q:
        for r in range(first, npass[t], stride):
            assert p0 + r not in words
            words.add(p0 + r)
    assert len(words) == nprog == sum(npass)
    if mode == 1:
        assert npipe == len(npass)
    else:
        assert all(stride == 1 and first == 0 for t, _, first, stride in q if t >= npipe)
