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


def border_thread(P, p, own, cb, sid, rs, n_own_slots, queued):
    """One border position of k_merge_2d's pair loop: staged neighbour p + d for each connected
    offset d; skipped when the node was just paired by this position (lastB) or when the position
    before, of the same own node, touches the same staged run; else the local filter decides."""
    ja = own[p]
    if ja < 0:
        return
    prev_cb = cb[p - 1] if p > 0 and own[p - 1] == ja else 0
    last_b = None
    for d in (-1, 0, 1):
        if not (cb[p] >> (d + 1)) & 1:
            continue
        i = p + d
        n_b = sid[i]
        if n_b == last_b:
            continue
        if any((prev_cb >> (dp + 1)) & 1 and rs[p - 1 + dp] == rs[i] for dp in (-1, 0, 1)):
            continue
        res = []
        yield from smerge_joined(P, ja, n_own_slots + rs[i], res)
        if res[0]:
            queued.append((1000 + ja, n_b))
        last_b = n_b


@pytest.mark.parametrize("seed", range(300))
def test_border_pairs_with_the_previous_position_rule(seed):
    """Every connected (own node, staged node) pair along a border is implied by the queued pairs
    when pairs covered by the previous position are skipped."""
    rng = random.Random(seed + 77)
    n_pos = rng.randint(2, 40)
    n_own_nodes, n_nodes = rng.randint(1, 6), rng.randint(1, 8)
    # own nodes along the border in runs (-1: empty), staged node ids in runs, staged index = position
    own, sid = [], []
    while len(own) < n_pos:
        own += [rng.choice([-1] + list(range(n_own_nodes)))] * rng.randint(1, 5)
    while len(sid) < n_pos + 1:
        sid += [rng.randrange(n_nodes)] * rng.randint(1, 5)
    own, sid = own[:n_pos], sid[:n_pos + 1]
    rs = [0] * len(sid)                              # staged run starts (same id, consecutive)
    for i in range(1, len(sid)):
        rs[i] = rs[i - 1] if sid[i] == sid[i - 1] else i
    cb = []
    for p in range(n_pos):
        m = 0
        for d in (-1, 0, 1):
            i = p + d
            if own[p] >= 0 and 0 <= i < len(sid) and rng.random() < 0.6:
                m |= 1 << (d + 1)
        cb.append(m)
    P = list(range(n_own_nodes + len(sid)))
    for i in range(len(sid)):
        P[n_own_nodes + i] = n_own_nodes + rs[i]
    queued = []
    run([border_thread(P, p, own, cb, sid, rs, n_own_nodes, queued) for p in range(n_pos)], rng)
    for p in range(n_pos):
        for d in (-1, 0, 1):
            if (cb[p] >> (d + 1)) & 1:
                assert connected(queued, 1000 + own[p], sid[p + d]), (p, d)
