"""Concurrent calls on ONE plan.

ft_b200_execute_dev and ft_b200_execute_sphv_dev take their scratch matrix, the rotation
kernel's work counter and the pass pipeline's progress words per call from a stream-ordered
memory pool, so several threads may drive one sph, tri or disk plan on several streams at
once.  Every result must be bit for bit the one a single thread gets calling the plan in turn
(the kernels do the same arithmetic whatever else runs).  The host-pointer ft_execute_* calls
on one plan share its staging buffer and stream and wait for each other: run from two threads
they must give the sequential results as well.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [("sph", (), 512), ("tri", (0.0, 0.0, 0.0), 384), ("disk", (0.0, 0.0), 256)]
OPS = [(True, "N"), (False, "N"), (True, "T"), (False, "T")]


@pytest.fixture(scope="module")
def env():
    import torch
    import fasttransforms_b200 as ft
    torch.cuda.set_device(0)
    return ft, torch


def make_plan(ft, kind, n, params):
    return {"sph": ft.plan_sph2fourier, "tri": ft.plan_tri2cheb, "disk": ft.plan_disk2cxf}[kind](n, *params)


def fields(ft, kind, n, count, seed):
    rand = {"sph": ft.sphrand, "tri": ft.trirand, "disk": ft.diskrand}[kind]
    return [np.asfortranarray(rand(n, seed + i)) for i in range(count)]


def run_dev(ft, torch, P, A, ops, stream):
    """Every op in turn on a device copy of A, enqueued on stream; the result on the host."""
    n, M = A.shape
    with torch.cuda.stream(stream):
        d = torch.from_numpy(A.ravel(order="F").copy()).cuda()
        for fw, tr in ops:
            ft.execute_dev(P, fw, tr, d.data_ptr(), n, M, stream.cuda_stream)
        out = d.cpu()
    stream.synchronize()
    return out.numpy().reshape((n, M), order="F")


@pytest.mark.parametrize("kind,params,n", CASES)
def test_device_calls_from_two_threads(env, kind, params, n):
    ft, torch = env
    P = make_plan(ft, kind, n, params)
    A = fields(ft, kind, n, 6, 20261204)
    streams = [torch.cuda.Stream() for _ in range(2)]
    # one thread, in turn: the reference results (the first call also fixes the autotuned shape)
    want = [run_dev(ft, torch, P, a, OPS, streams[0]) for a in A]
    got = [None] * len(A)
    errors = []
    start = threading.Barrier(2)

    def worker(w):
        try:
            start.wait()
            for rep in range(3):   # several rounds, so that the two streams' calls overlap
                for i in range(w, len(A), 2):
                    got[i] = run_dev(ft, torch, P, A[i], OPS, streams[w])
        except Exception as e:   # reported on the main thread
            errors.append(e)

    th = [threading.Thread(target=worker, args=(w,)) for w in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for i in range(len(A)):
        assert np.array_equal(got[i], want[i]), (kind, i)


def test_sphv_device_calls_from_two_threads(env):
    ft, torch = env
    n = 256
    P = ft.plan_sph2fourier(n)
    M = 2 * n - 1
    rng = np.random.default_rng(7)
    A = [np.asfortranarray(rng.standard_normal((n, M))) for _ in range(4)]
    streams = [torch.cuda.Stream() for _ in range(2)]

    def run(a, s):
        with torch.cuda.stream(s):
            d = torch.from_numpy(a.ravel(order="F").copy()).cuda()
            ft.execute_sphv_dev(P, True, "N", d.data_ptr(), n, M, s.cuda_stream)
            ft.execute_sphv_dev(P, False, "N", d.data_ptr(), n, M, s.cuda_stream)
            out = d.cpu()
        s.synchronize()
        return out.numpy().reshape((n, M), order="F")

    want = [run(a, streams[0]) for a in A]
    got = [None] * len(A)
    th = [threading.Thread(target=lambda w=w: [got.__setitem__(i, run(A[i], streams[w])) for i in range(w, len(A), 2)])
          for w in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(len(A)):
        assert np.array_equal(got[i], want[i]), i


def test_host_calls_from_two_threads(env):
    ft, torch = env
    n = 256
    P = ft.plan_sph2fourier(n)
    A = fields(ft, "sph", n, 4, 99)
    want = []
    for a in A:
        b = a.copy(order="F")
        ft.execute_sph2fourier("N", P, b)
        ft.execute_fourier2sph("N", P, b)
        want.append(b)
    got = [a.copy(order="F") for a in A]

    def worker(w):
        for i in range(w, len(A), 2):
            ft.execute_sph2fourier("N", P, got[i])
            ft.execute_fourier2sph("N", P, got[i])

    th = [threading.Thread(target=worker, args=(w,)) for w in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(len(A)):
        assert np.array_equal(got[i], want[i]), i
