"""Continuous batching (femgpu_stream_*): requests that arrive while others run are admitted into
free slots of the device loop, each solved as the batch solves it.

The batch's own solve (femgpu_batch_solve, every pair from x = 0) is the reference here: each
streamed request's solution must equal it bit for bit, whether it ran alone in the loop or
among many others (each slot's arithmetic reads only its own data), and the loop must have
packed several requests into its iterations. The batch solve itself is checked against the
oracle's direct solutions in tests/test_gpu_batch.py.
"""
import time

import numpy as np
import pytest

import femahoy_b200 as fg
from femahoy_b200.batch import Batch, Stream
from test_gpu_batch import _direct, _member, _rel

pytestmark = pytest.mark.gpu


def _members(seed, count=5):
    rng = np.random.default_rng(seed)
    return [_member(rng, hi=(24, 3, 3)) for _ in range(count)]


def _make(members, precision):
    b = Batch([m[1] for m in members], [m[3] for m in members], 4, precision=precision,
              options=fg.Options(precision=precision, coarsest=256))
    return b.with_tol(1e-10)


@pytest.mark.parametrize("precision", [fg.MIXED, fg.FP64])
def test_stream_equals_the_batch_alone_and_in_a_mix(precision):
    members = _members(21)
    ref, _ = _make(members, precision).solve([m[2] for m in members])
    stream = Stream(_make(members, precision))
    # 1 request alone in the loop. The true residual is held to tol with the batch tests' 20 %
    # slack: at 1e-10 the recurrence of these systems drifts from b - Ax by up to a few percent,
    # which the at most 3 restarts from x do not always remove (the batch solve gives the same).
    x, res = stream.wait(stream.submit(2, members[2][2][:, 1]))
    assert res.status == 0 and res.true_residual <= 1.2e-10
    assert np.array_equal(x.view(np.uint64), ref[2][:, 1].view(np.uint64))
    # Every right side of every system, submitted while earlier ones run, 2 systems with more
    # requests than slots (they queue for a free slot).
    jobs = []
    order = [(k, r) for r in range(4) for k in range(len(members))]
    order += [(0, 3), (0, 0), (4, 2)]
    for i, (k, r) in enumerate(order):
        jobs.append((k, r, stream.submit(k, members[k][2][:, r])))
        if i % 5 == 4:
            time.sleep(0.002)
    for k, r, t in jobs:
        x, res = stream.wait(t)
        assert res.status == 0 and res.true_residual <= 1.2e-10, (k, r, res.true_residual)
        assert np.array_equal(x.view(np.uint64), ref[k][:, r].view(np.uint64)), (k, r)
    loops, served = stream.counts()
    assert served > loops, "the loop packed several requests into its iterations"
    stream.close()


def test_stream_against_the_direct_solutions():
    """The streamed solutions of 3 systems against the oracle's multifrontal Cholesky."""
    members = _members(8, count=3)
    stream = Stream(_make(members, fg.MIXED))
    tickets = [(k, r, stream.submit(k, members[k][2][:, r])) for k in range(3) for r in range(4)]
    direct = [_direct(m[0], m[2]) for m in members]
    for k, r, t in tickets:
        x, _ = stream.wait(t)
        assert _rel(x, direct[k][:, r]) <= 1e-6
    stream.close()


def test_stream_refuses_the_batch_solve_and_bad_requests():
    members = _members(3, count=2)
    b = _make(members, fg.MIXED)
    stream = Stream(b)
    with pytest.raises(fg.FemError, match="serves a stream"):
        b.solve([m[2] for m in members])
    with pytest.raises(fg.FemError, match="no such system"):
        stream.submit(5, np.zeros(10))
    # A zero right side gives x = 0 at once.
    x, res = stream.wait(stream.submit(1, np.zeros(stream.rows(1))))
    assert not x.any() and res.iterations == 0
    stream.close()
