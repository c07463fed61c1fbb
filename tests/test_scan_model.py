"""Interleaving model of the single-pass segment scan (labeling_b200/csrc/be_scan.cuh:
segscan_lb_chunk).  Chunks take tickets in the order their CTAs start, publish their own sum
(state 1), look back over earlier chunks 32 at a time -- a lane per chunk, each status word read on
its own, so a round sees a mix of old and new states -- until the nearest inclusive prefix
(state 2), and publish their inclusive prefix.  Status words carry the launch epoch, and words left
by an earlier launch read as not ready.  A seeded random scheduler interleaves every chunk's steps
after the tickets are taken; every schedule must give each chunk the exact sum of the chunks before
it, and no look-back may wait on a chunk that has not started (it could not end)."""
import random

import pytest


def chunk(c, total, st, ep, result, started):
    started.add(c)
    yield
    st[c] = (ep, 1, total)                       # this chunk's sum
    yield
    excl, base = 0, 0
    while c - 1 - base >= 0:
        states, values = [], []
        for lane in range(32):                   # the lanes' loads, one step each
            j = c - 1 - base - lane
            if j >= 0:
                e, s, v = st[j]
                states.append(s if e == ep else 0)
                values.append(v)
                yield
            else:
                states.append(2)                 # before chunk 0: an empty inclusive prefix
                values.append(0)
        incl = [lane for lane in range(32) if states[lane] == 2]
        stop = incl[0] if incl else 31
        need = range(stop + 1)
        if any(states[lane] == 0 for lane in need):
            for lane in need:                    # a spin may only wait on chunks already started
                j = c - 1 - base - lane
                if j >= 0 and states[lane] == 0:
                    assert j in started
            yield
            continue
        excl += sum(values[lane] for lane in range(stop + 1) if c - 1 - base - lane >= 0)
        if incl:
            break
        base += 32
    st[c] = (ep, 2, excl + total)                # inclusive prefix
    result[c] = excl
    yield


def run_scan(totals, rng, stale):
    n = len(totals)
    ep = 7
    st = [(ep - 1, 2, 999999) if stale else (0, 0, 0) for _ in range(n)]   # words of an earlier launch
    result, started = {}, set()
    pending = [chunk(c, totals[c], st, ep, result, started) for c in range(n)]
    live = []
    while pending or live:
        # a chunk's CTA starts (and takes its ticket) only after all earlier tickets were taken
        if pending and (not live or rng.random() < 0.3):
            g = pending.pop(0)
            next(g)
            live.append(g)
            continue
        i = rng.randrange(len(live))
        try:
            next(live[i])
        except StopIteration:
            live[i] = live[-1]
            live.pop()
    return result


@pytest.mark.parametrize("seed", range(60))
def test_lookback_gives_exact_prefixes(seed):
    rng = random.Random(seed)
    n = rng.randint(1, 100)
    totals = [rng.randint(0, 5000) for _ in range(n)]
    result = run_scan(totals, rng, stale=seed % 2 == 1)
    acc = 0
    for c in range(n):
        assert result[c] == acc
        acc += totals[c]
