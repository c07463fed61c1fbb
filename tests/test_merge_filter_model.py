"""Interleaving model of the merge kernels' CTA-local filter (labeling_b200/csrc/be_common.cuh:
smerge_joined; k_merge_2d / k_merge_3d in be_uf2d_impl.cuh / be_uf3d.cu).  A tile's own border
nodes and the staged border positions of its neighbours are elements of a shared-memory union-find
(smaller index wins, atomicMin, path halving); staged positions of one neighbour node that touch
start as one element (each points at its run's first position).  Every connected (own node,
staged position) pair calls smerge_joined, and only a call that reports a join queues the pair of
global node ids for the global union-find.  The claim that makes the filter safe: local
connectivity never runs ahead of the queued global unions, so at the end every pair seen -- queued
or filtered -- is implied by the queued pairs.  Each shared access is one step of a generator and
a seeded random scheduler interleaves all the calls."""
import random

import pytest


def sfind(P, a):
    p = P[a]
    yield
    while p != a:
        g = P[p]
        yield
        if g != p:
            P[a] = g
            yield
        a, p = p, g
    return a


def smerge_joined(P, a, b, out):
    changed = False
    while True:
        a = yield from sfind(P, a)
        b = yield from sfind(P, b)
        if a == b:
            out.append(changed)
            return
        if a < b:
            old = P[b]                       # atomicMin, one step
            P[b] = min(old, a)
            yield
            if old == b:
                out.append(True)
                return
            changed |= old > a
            b = old
        else:
            old = P[a]
            P[a] = min(old, b)
            yield
            if old == a:
                out.append(True)
                return
            changed |= old > b
            a = old


def pair_thread(P, own_elem, staged_elem, g_own, g_staged, queued):
    res = []
    yield from smerge_joined(P, own_elem, staged_elem, res)
    if res[0]:
        queued.append((g_own, g_staged))


def run(threads, rng):
    live = list(threads)
    while live:
        i = rng.randrange(len(live))
        try:
            next(live[i])
        except StopIteration:
            live[i] = live[-1]
            live.pop()


def connected(pairs, a, b):
    adj = {}
    for x, y in pairs:
        adj.setdefault(x, set()).add(y)
        adj.setdefault(y, set()).add(x)
    seen, todo = {a}, [a]
    while todo:
        x = todo.pop()
        if x == b:
            return True
        for y in adj.get(x, ()):
            if y not in seen:
                seen.add(y)
                todo.append(y)
    return a == b


@pytest.mark.parametrize("seed", range(300))
def test_filtered_pairs_are_implied_by_queued_ones(seed):
    rng = random.Random(seed)
    n_own = rng.randint(1, 12)
    n_staged = rng.randint(1, 40)
    n_nodes = rng.randint(1, 10)                     # the neighbours' global nodes
    # staged positions: runs of equal node ids (each run points at its first position)
    sid, k = [], 0
    while k < n_staged:
        length = min(n_staged - k, rng.randint(1, 6))
        sid += [rng.randrange(n_nodes)] * length
        k += length
    P = list(range(n_own + n_staged))
    for k in range(1, n_staged):
        if sid[k] == sid[k - 1]:
            P[n_own + k] = P[n_own + k - 1]
    g_own = [1000 + i for i in range(n_own)]          # global ids of the tile's own nodes
    pairs = [(rng.randrange(n_own), rng.randrange(n_staged)) for _ in range(rng.randint(1, 60))]
    queued = []
    run([pair_thread(P, i, n_own + k, g_own[i], sid[k], queued) for i, k in pairs], rng)
    for i, k in pairs:
        assert connected(queued, g_own[i], sid[k]), (i, k, sid[k], queued)
