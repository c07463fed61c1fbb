"""Interleaving model of the global union-find the merge kernels run (labeling_b200/csrc/
be_common.cuh: gunion_keyed, gfind_jump).  Each shared-memory access of a union or a flatten is one
step of a Python generator, and a seeded random scheduler interleaves many of them, as the GPU's
threads do.  Entries are (key of the parent, parent) pairs, read, written and compared-and-swapped
whole, as the kernels' 64-bit words.  On random graphs, on long paths whose keys rise along the
path (the spiral's and serpentine's worst case) and on stars, every schedule must end with:

* the partition of the graph's connected components,
* each component rooted at its smallest key (the first pixel that numbers it canonically),
* the "linked" callback called exactly once for every other node of a component -- the kernels
  clear that node's root bit and segment count there, so a miss or a repeat would miscount,
* keys strictly decreasing along every parent path,

and the pointer-jumping flatten must leave every node pointing straight at its root."""
import random

import pytest


def union(mem, a, b, linked):
    """gunion_keyed: Rem's interleaved climb with path halving, link by CAS."""
    ea = mem[a]
    yield
    eb = mem[b]
    yield
    while True:
        if ea[1] == eb[1]:
            return                                   # same parent: one set
        if ea[0] < eb[0]:                            # climb on the side with the larger parent key
            a, b, ea, eb = b, a, eb, ea
        pa = ea[1]
        if pa == a:                                  # a root: link it under b's parent
            old = mem[a]                             # compare-and-swap, one step
            if old == ea:
                mem[a] = eb
                linked.append(ea[0])
                yield
                return
            ea = old
            yield
            eb = mem[b]
            yield
            continue
        ga = mem[pa]
        yield
        if ga[1] != pa:
            mem[a] = ga                              # path halving
            yield
        a, ea = pa, ga


def jump(mem, x):
    """gfind_jump and the store of the root's entry (flatten_tile_nodes / link_tile_nodes)."""
    p = mem[x][1]
    yield
    if p == x:
        return
    while True:
        ep = mem[p]
        yield
        if ep[1] == p:
            break
        mem[x] = ep                                  # only this node's own entry is written
        yield
        p = ep[1]
    mem[x] = mem[p]
    yield


def run(threads, rng):
    live = [t for t in threads]
    while live:
        i = rng.randrange(len(live))
        try:
            next(live[i])
        except StopIteration:
            live[i] = live[-1]
            live.pop()


def components(n, edges):
    parent = list(range(n))

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for a, b in edges:
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[ra] = rb
    return [find(x) for x in range(n)]


def root_of(mem, x):
    while mem[x][1] != x:
        x = mem[x][1]
    return x


def check(n, edges, keys, seed):
    rng = random.Random(seed)
    mem = {x: (keys[x], x) for x in range(n)}
    linked = []
    run([union(mem, a, b, linked) for a, b in edges], rng)
    # keys strictly decrease along every parent path, and every entry names its parent's key
    for x in range(n):
        k, p = mem[x]
        assert k == keys[p]
        assert p == x or keys[p] < keys[x]
    comp = components(n, edges)
    groups = {}
    for x in range(n):
        groups.setdefault(comp[x], []).append(x)
    for members in groups.values():
        want_root = min(members, key=lambda x: keys[x])
        for x in members:
            assert root_of(mem, x) == want_root
    expected_links = sorted(keys[x] for members in groups.values() for x in members
                            if x != min(members, key=lambda y: keys[y]))
    assert sorted(linked) == expected_links
    roots = {x: root_of(mem, x) for x in range(n)}
    run([jump(mem, x) for x in range(n)], rng)
    for x in range(n):
        assert mem[x][1] == roots[x] and mem[x][0] == keys[roots[x]]


@pytest.mark.parametrize("seed", range(200))
def test_random_graphs(seed):
    rng = random.Random(seed)
    n = rng.randint(2, 60)
    keys = rng.sample(range(10 * n), n)
    m = rng.randint(1, 2 * n)
    edges = [(rng.randrange(n), rng.randrange(n)) for _ in range(m)]
    check(n, edges, keys, seed + 1000)


@pytest.mark.parametrize("seed", range(40))
def test_long_paths_with_rising_keys(seed):
    rng = random.Random(seed)
    n = rng.randint(20, 120)
    keys = list(range(n)) if seed % 2 == 0 else list(range(n, 0, -1))
    # one path through all nodes, edges in a random order, some repeated
    edges = [(i, i + 1) for i in range(n - 1)]
    edges += rng.sample(edges, min(len(edges), 10))
    rng.shuffle(edges)
    check(n, edges, keys, seed + 2000)


@pytest.mark.parametrize("seed", range(20))
def test_stars_and_cliques(seed):
    rng = random.Random(seed)
    n = rng.randint(10, 40)
    keys = rng.sample(range(1000), n)
    hub = rng.randrange(n)
    edges = [(hub, x) for x in range(n) if x != hub]
    edges += [(rng.randrange(n), rng.randrange(n)) for _ in range(n)]
    rng.shuffle(edges)
    check(n, edges, keys, seed + 3000)
