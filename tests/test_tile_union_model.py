"""Interleaving model of the in-tile union-find the tile kernels run in shared memory
(labeling_b200/csrc/be_uf2d_impl.cuh: efind_e / eunion and the root walk of phase C; the 3D kernel
has the same efind3_e / eunion3).  Entries are (slot << 12) | parent; a root holds its own slot and
index, a forest link (a run's first link into the row above, whose slots are all smaller) holds
slot 0 so that no atomicMin changes it; a union lowers a root's entry with atomicMin, and finds
halve paths with plain stores.  Each shared-memory access is one step of a Python generator and a
seeded random scheduler interleaves the unions of all lanes; then every run start walks to its
root (read-only) and stores the root's entry in its own, again interleaved.  Every schedule must
leave each run pointing at the run with the smallest slot of its component (the run holding the
component's first pixel), with that run's slot in the entry."""
import random

import pytest

IDX = 0xFFF


def efind_e(P, x):
    v = P[x]
    yield
    while (v & IDX) != x:
        y = v & IDX
        vg = P[y]
        yield
        if (vg & IDX) != y:
            P[x] = vg
            yield
        x, v = y, vg
    return x, v


def eunion(P, a, b):
    while True:
        a, ea = yield from efind_e(P, a)
        b, eb = yield from efind_e(P, b)
        if a == b:
            return
        if ea < eb:
            old = P[b]                       # atomicMin, one step
            P[b] = min(old, ea)
            yield
            if (old & IDX) == b:
                return
            b = old & IDX
        else:
            old = P[a]
            P[a] = min(old, eb)
            yield
            if (old & IDX) == a:
                return
            a = old & IDX


def walk(P, x):
    root, ev = x, P[x]
    yield
    while (ev & IDX) != root:
        root = ev & IDX
        ev = P[root]
        yield
    if root != x:
        P[x] = ev
        yield


def run(threads, rng):
    live = list(threads)
    while live:
        i = rng.randrange(len(live))
        try:
            next(live[i])
        except StopIteration:
            live[i] = live[-1]
            live.pop()


def check(n, forest, edges, slots, seed):
    """forest: node -> parent with a smaller slot (or absent); edges: unions."""
    rng = random.Random(seed)
    P = {x: ((slots[x] << 12) | x) if x not in forest else forest[x] for x in range(n)}
    run([eunion(P, a, b) for a, b in edges], rng)
    run([walk(P, x) for x in range(n)], rng)
    # expected components over forest links and union edges
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in list(forest.items()) + edges:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[ra] = rb
    best = {}
    for x in range(n):
        r = find(x)
        if r not in best or slots[x] < slots[best[r]]:
            best[r] = x
    for x in range(n):
        want = best[find(x)]
        assert P[x] & IDX == want, (x, P[x] & IDX, want)
        assert P[x] >> 12 == slots[want]


def case(rng, n, n_edges):
    slots = rng.sample(range(1, 8 * n), n)          # slot 0 is the forest links' key
    order = sorted(range(n), key=lambda x: slots[x])
    forest = {}
    for i, x in enumerate(order):
        if i and rng.random() < 0.6:                 # a parent among the runs with smaller slots
            forest[x] = order[rng.randrange(i)]
    edges = [(rng.randrange(n), rng.randrange(n)) for _ in range(n_edges)]
    return slots, forest, edges


@pytest.mark.parametrize("seed", range(200))
def test_random_forests_and_unions(seed):
    rng = random.Random(seed)
    n = rng.randint(2, 70)
    slots, forest, edges = case(rng, n, rng.randint(0, 2 * n))
    check(n, forest, edges, slots, seed + 5000)


@pytest.mark.parametrize("seed", range(40))
def test_deep_forest_chains(seed):
    """Vertical chains (every run's parent the run just above), joined by unions at their ends,
    as a 1-pixel spiral or serpentine gives them."""
    rng = random.Random(seed)
    chains, depth = rng.randint(2, 6), rng.randint(5, 25)
    n = chains * depth
    slots = [0] * n
    forest = {}
    for c in range(chains):
        for d in range(depth):
            x = c * depth + d
            slots[x] = 1 + d * chains + c             # raster order: row d, column c
            if d:
                forest[x] = x - 1
    edges = []
    for c in range(chains - 1):
        a = c * depth + (depth - 1 if c % 2 == 0 else 0)
        edges.append((a, (c + 1) * depth + rng.randrange(depth)))
    edges += [(rng.randrange(n), rng.randrange(n)) for _ in range(rng.randint(0, 5))]
    rng.shuffle(edges)
    check(n, forest, edges, slots, seed + 6000)
