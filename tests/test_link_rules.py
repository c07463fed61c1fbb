"""The tile kernels' run and link rules, restated on whole block rows and checked against the oracle
(labeling_b200/csrc/be_uf2d_impl.cuh, k_tile_local_2d phases A and B).  Blocks are 2x2 pixels; a
block row's four pixel classes (top-left, top-right, bottom-left, bottom-right) are bit sets, so
runs of horizontally joined blocks, run starts and the N / NW / NE links to the row above are bit
operations, and a link is dropped when an earlier link (further left, or N before NW / NE at the
same block) joins the same two runs.  Uniting the runs over the kept links must give exactly the
8-connected components of the image: a rule that dropped a needed link would split a component,
and the GPU kernel makes the same decisions word by word.  The 3D kernel (be_uf3d.cu,
k_tile_local_3d phases A and B) is restated the same way: rows along d2 with eight voxel-class bit
sets, 26-connected face tests toward the four preceding rows, the same drop rules, against the
oracle's 26-connected components."""
import numpy as np
import pytest

from labeling_b200 import workloads as W
from oracle import oracle as O


def bits(row):
    """Bit set of a boolean row: bit k = row[k]."""
    v = 0
    for k in np.flatnonzero(row):
        v |= 1 << int(k)
    return v


def hibit_le(mask, k):
    """Highest set bit of mask at or below k."""
    m = mask & ((2 << k) - 1)
    return m.bit_length() - 1


def block_partition(img):
    fg = img > 0
    h, w = fg.shape
    hb, wb = (h + 1) // 2, (w + 1) // 2
    pad = np.zeros((2 * hb, 2 * wb), bool)
    pad[:h, :w] = fg
    TL, TR, BL, BR = pad[0::2, 0::2], pad[0::2, 1::2], pad[1::2, 0::2], pad[1::2, 1::2]
    parent = {}

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    def union(a, b):
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)

    prev = None
    starts = []
    for r in range(hb):
        tl, tr, bl, br = bits(TL[r]), bits(TR[r]), bits(BL[r]), bits(BR[r])
        lw, rw, tw = tl | bl, tr | br, tl | tr
        fw = tw | bl | br
        hc = rw & (lw >> 1)                 # block k joined to k + 1
        hl = hc << 1                        # block k joined to k - 1
        s = fw & ~hl                        # run starts
        starts.append(s)
        for k in range(wb):
            if (s >> k) & 1:
                parent[r * wb + k] = r * wb + k
        if prev is not None:
            ubl, ubr, uhc = prev
            uhl = uhc << 1
            n = tw & (ubl | ubr)
            nw = tl & (ubr << 1)
            ne = tr & (ubl >> 1)
            nsh, nesh = n << 1, ne << 1
            nm = n & ~(hl & ((nsh & uhl) | nesh))
            nwm = nw & ~((n & uhl) | (hl & nsh))
            nem = ne & ~((n & uhc) | (hl & nesh & uhc))
            for k in range(wb):
                a = r * wb + hibit_le(s, k)
                for m, dk in ((nm, 0), (nwm, -1), (nem, 1)):
                    if (m >> k) & 1:
                        union(a, (r - 1) * wb + hibit_le(starts[r - 1], k + dk))
        prev = (bl, br, hc)
    lab = np.full((hb, wb), -1, np.int64)
    for r in range(hb):
        fw_r = TL[r] | TR[r] | BL[r] | BR[r]
        for k in np.flatnonzero(fw_r):
            lab[r, k] = find(r * wb + hibit_le(starts[r], int(k)))
    return lab


def assert_same_partition(img):
    lab = block_partition(img)
    ref, _ = O.ccl2d(img)
    hb, wb = lab.shape
    pad = np.zeros((2 * hb, 2 * wb), np.int64)
    pad[:img.shape[0], :img.shape[1]] = ref
    # the oracle's label of each block: any of its foreground pixels (a 2x2 block is connected)
    blk = np.maximum(np.maximum(pad[0::2, 0::2], pad[0::2, 1::2]), np.maximum(pad[1::2, 0::2], pad[1::2, 1::2]))
    fg = lab >= 0
    assert np.array_equal(fg, blk > 0)
    pairs = set(zip(lab[fg].tolist(), blk[fg].tolist()))
    # a bijection between the restated sets and the oracle's components
    assert len(pairs) == len({a for a, _ in pairs}) == len({b for _, b in pairs})


@pytest.mark.parametrize("seed", range(120))
def test_random_images(seed):
    rng = np.random.default_rng(seed)
    h, w = int(rng.integers(1, 90)), int(rng.integers(1, 130))
    p = float(rng.uniform(0.05, 0.95))
    assert_same_partition(W.bernoulli((h, w), p, seed))


@pytest.mark.parametrize("shape", [(64, 96), (63, 97), (40, 200)])
def test_paths_and_patterns(shape):
    h, w = shape
    assert_same_partition(W.serpentine(h, w))
    assert_same_partition(W.spiral(h, w))
    yy, xx = np.mgrid[:h, :w]
    assert_same_partition(((yy + xx) % 2 * 255).astype(np.uint8))        # checkerboard: diagonals only
    assert_same_partition((((yy // 2) + (xx // 2)) % 2 * 255).astype(np.uint8))
    assert_same_partition(W.disks(h, w, 6, 2, 12, 0.05, seed=3))


# ---- 3D: rows along d2, 26-connectivity, links to the four preceding rows ---------------------

def face_word(c, dx, dy, dz):
    """OR of the voxel classes v = 4i + 2j + k on the block side facing (dx, dy, dz)."""
    r = 0
    for v in range(8):
        i, j, k = v >> 2, (v >> 1) & 1, v & 1
        if (dx < 0 and i) or (dx > 0 and not i) or (dy < 0 and j) or (dy > 0 and not j) or \
           (dz < 0 and k) or (dz > 0 and not k):
            continue
        r |= c[v]
    return r


def block_partition_3d(vol):
    fg = vol > 0
    d0, d1, d2 = fg.shape
    n0, n1, n2 = (d0 + 1) // 2, (d1 + 1) // 2, (d2 + 1) // 2
    pad = np.zeros((2 * n0, 2 * n1, 2 * n2), bool)
    pad[:d0, :d1, :d2] = fg
    cls = [pad[v >> 2::2, (v >> 1) & 1::2, v & 1::2] for v in range(8)]   # [n0][n1][n2] each
    rows = {}
    for b0 in range(n0):
        for b1 in range(n1):
            c = [bits(cls[v][b0, b1]) for v in range(8)]
            hz = face_word(c, 0, 0, 1) & (face_word(c, 0, 0, -1) >> 1)
            fw = 0
            for x in c:
                fw |= x
            rows[(b0, b1)] = (c, hz, fw & ~(hz << 1), fw)
    parent = {}

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    def key(b0, b1, k):
        return (b0 * n1 + b1) * n2 + k

    for (b0, b1), (_, _, s, _) in rows.items():
        for k in range(n2):
            if (s >> k) & 1:
                parent[key(b0, b1, k)] = key(b0, b1, k)
    for (b0, b1), (c, hz, s, fw) in rows.items():
        hl = hz << 1
        for nr in range(4):
            dx, dy = (-1, nr - 1) if nr < 3 else (0, -1)
            r0, r1 = b0 + dx, b1 + dy
            if r0 < 0 or r1 < 0 or r1 >= n1:
                continue
            u, uhz, us, _ = rows[(r0, r1)]
            uhl = uhz << 1
            a0, am, ap = face_word(c, dx, dy, 0), face_word(c, dx, dy, -1), face_word(c, dx, dy, 1)
            bb0, bm, bp = face_word(u, -dx, -dy, 0), face_word(u, -dx, -dy, 1), face_word(u, -dx, -dy, -1)
            n0_ = a0 & bb0
            nw = am & (bm << 1)
            ne = ap & (bp >> 1)
            nsh, nesh = n0_ << 1, ne << 1
            nm = n0_ & ~(hl & ((nsh & uhl) | nesh))
            nwm = nw & ~((n0_ & uhl) | (hl & nsh))
            nem = ne & ~((n0_ & uhz) | (hl & nesh & uhz))
            for k in range(n2):
                a = key(b0, b1, hibit_le(s, k))
                for m, dk in ((nm, 0), (nwm, -1), (nem, 1)):
                    if (m >> k) & 1:
                        ra, rb = find(a), find(key(r0, r1, hibit_le(us, k + dk)))
                        if ra != rb:
                            parent[max(ra, rb)] = min(ra, rb)
    lab = np.full((n0, n1, n2), -1, np.int64)
    for (b0, b1), (_, _, s, fw) in rows.items():
        for k in range(n2):
            if (fw >> k) & 1:
                lab[b0, b1, k] = find(key(b0, b1, hibit_le(s, k)))
    return lab


def assert_same_partition_3d(vol):
    lab = block_partition_3d(vol)
    ref, _ = O.ccl3d(vol)
    n0, n1, n2 = lab.shape
    pad = np.zeros((2 * n0, 2 * n1, 2 * n2), np.int64)
    pad[:vol.shape[0], :vol.shape[1], :vol.shape[2]] = ref
    blk = np.zeros(lab.shape, np.int64)
    for v in range(8):
        blk = np.maximum(blk, pad[v >> 2::2, (v >> 1) & 1::2, v & 1::2])
    fg = lab >= 0
    assert np.array_equal(fg, blk > 0)
    pairs = set(zip(lab[fg].tolist(), blk[fg].tolist()))
    assert len(pairs) == len({a for a, _ in pairs}) == len({b for _, b in pairs})


@pytest.mark.parametrize("seed", range(60))
def test_random_volumes(seed):
    rng = np.random.default_rng(seed + 500)
    shape = tuple(int(x) for x in rng.integers(1, 20, size=3))
    p = float(rng.uniform(0.05, 0.6))
    assert_same_partition_3d(W.bernoulli(shape, p, seed))


def test_volume_diagonals_and_planes():
    zz, yy, xx = np.mgrid[:12, :14, :18]
    assert_same_partition_3d((((zz + yy + xx) % 2) * 255).astype(np.uint8))              # corners only
    assert_same_partition_3d(((((zz // 2) + (yy // 2) + (xx // 2)) % 2) * 255).astype(np.uint8))
    assert_same_partition_3d(((zz % 3 == 0) * 255).astype(np.uint8))                        # planes
