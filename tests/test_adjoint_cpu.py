"""The binomial checkpoint schedule of the adjoint (host logic, no GPU): every step is
reversed exactly once, in order N-1 .. 0, from its own state; no more snapshots are
live than allowed; the forward steps match the binomial optimum."""
import numpy as np
import pytest

from geoswe_b200.adjoint import Treeverse, binomial_beta, interp_weights, snapshot_chain, treeverse_split


def _run(N, S, pre_stored=True):
    snaps = {0: 0}
    cur = {"n": None}

    def store(n):
        assert cur["n"] == n
        snaps[n] = n

    def restore(n):
        cur["n"] = snaps[n]

    def advance(n0, n1):
        assert cur["n"] == n0
        cur["n"] = n1

    def free(n):
        snaps.pop(n)

    def reverse(n):
        assert cur["n"] == n, (cur["n"], n)

    chain = snapshot_chain(N, S) if pre_stored else []
    for m in chain:
        snaps[m] = m
    tv = Treeverse(N, S, store, restore, advance, free, reverse, stored=chain)
    tv.run()
    return tv


@pytest.mark.parametrize("N,S", [(1, 3), (2, 1), (7, 2), (100, 3), (200, 10), (1000, 20), (3000, 55), (50, 0)])
def test_every_step_reversed_once_in_order(N, S):
    tv = _run(N, S)
    assert tv.order == list(range(N - 1, -1, -1))
    assert tv.max_live <= S


@pytest.mark.parametrize("N,S", [(100, 3), (200, 10), (1000, 20), (3000, 55)])
def test_forward_steps_binomial_optimum(N, S):
    tv = _run(N, S)
    t = 0
    while binomial_beta(S, t) < N:
        t += 1
    optimum = t * N - binomial_beta(S + 1, t - 1)
    assert tv.forward_steps + N <= optimum + 1          # + the recording pass


def test_split_keeps_recomputation_count():
    for N in (10, 57, 300, 3000):
        for S in (1, 4, 55):
            m = treeverse_split(N, S)
            assert 1 <= m <= N - 1


def test_interp_weights_reproduce_numpy():
    rng = np.random.default_rng(0)
    xp = np.sort(rng.uniform(0, 100, 9))
    fp = rng.normal(size=9)
    t = np.concatenate([rng.uniform(-10, 110, 50), xp])
    assert np.allclose(interp_weights(t, xp) @ fp, np.interp(t, xp, fp), rtol=0, atol=1e-12)
