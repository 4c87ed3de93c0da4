"""Properties of the linear BVH that the full-IPC candidate search relies on,
checked on a Python restatement of its construction (Karras 2012, as
k_karras builds it over sorted unique 64-bit keys (Morton << 32 | index)).

- Every inner node's index is one end of its leaf range.  The chunked
  refit (k_refit) depends on this: a node whose range lies inside a block's
  chunk of leaves has its index there too, so the node's counter and box
  can live in that block's shared memory.
- The refit's chunked hand-over gives the same boxes as a plain bottom-up
  merge, in whatever order the threads arrive.
- A walk that tests both children at their parent (k_traverse) finds
  exactly the leaves whose boxes overlap the query box.
- The depth stays far below the traversal's stack of 96 entries.
- The bitonic network that sorts a query's candidate slice longer than 64
  in its warp's shared row (k_sort_query_slices) sorts every length up to
  2048.
"""
import numpy as np


def clz64(x):
    return 64 - int(x).bit_length()


def karras(keys):
    """child[i] = (left, right) with ~leaf for leaves; rng[i] = (lo, hi)."""
    n = len(keys)

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        return clz64(keys[i] ^ keys[j])

    child, rng = [], []
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) >= 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while lmax < 2 * n and delta(i, i + lmax * d) > dmin:
            lmax <<= 1
        l, t = 0, lmax >> 1
        while t >= 1:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t >>= 1
        j = i + l * d
        dnode = delta(i, j)
        s, t = 0, l
        while t > 1:
            t = (t + 1) >> 1
            if delta(i, i + (s + t) * d) > dnode:
                s += t
        gamma = i + s * d + (-1 if d < 0 else 0)
        lo, hi = min(i, j), max(i, j)
        left = ~gamma if lo == gamma else gamma
        right = ~(gamma + 1) if hi == gamma + 1 else gamma + 1
        child.append((left, right))
        rng.append((lo, hi))
    return child, rng


def sample_keys(rng, n, morton_bits):
    morton = rng.integers(0, 1 << morton_bits, size=n)
    return sorted(int(m) << 32 | i for i, m in enumerate(morton))


def leaf_boxes(rng, n):
    lo = rng.uniform(-1.0, 1.0, size=(n, 3))
    return np.hstack([lo, lo + rng.uniform(0.0, 0.2, size=(n, 3))])


def plain_refit(child, n, leaf):
    box = {}

    def rec(c):
        if c < 0:
            return leaf[~c]
        b0, b1 = rec(child[c][0]), rec(child[c][1])
        box[c] = np.hstack([np.minimum(b0[:3], b1[:3]), np.maximum(b0[3:], b1[3:])])
        return box[c]

    rec(0)
    return box


def chunked_refit(child, rng_, n, leaf, chunk, order):
    """k_refit's protocol run sequentially, the leaves' threads taken in
    `order`: a thread climbs while it is the second to arrive at a node;
    nodes inside its chunk count in the chunk's counters, the others in the
    device-wide ones."""
    parent = {}
    for i, (a, b) in enumerate(child):
        parent[a] = i
        parent[b] = i
    local_flags, global_flags, box, used_local = {}, {}, {}, set()
    for s in order:
        s0 = (s // chunk) * chunk
        last = min(s0 + chunk, n) - 1
        b = leaf[s].copy()
        frm, node, local = ~s, parent.get(~s, -1), True
        while node >= 0:
            c0, c1 = child[node]
            sib = c1 if c0 == frm else c0
            if local:
                lo, hi = rng_[node]
                local = lo >= s0 and hi <= last
            if local:
                assert s0 <= node <= last          # the node's shared-memory slot is inside the chunk
                key = (s0, node)
                local_flags[key] = local_flags.get(key, 0) + 1
                used_local.add(node)
                if local_flags[key] == 1:
                    break
            else:
                global_flags[node] = global_flags.get(node, 0) + 1
                if global_flags[node] == 1:
                    break
            o = leaf[~sib] if sib < 0 else box[sib]
            b = np.hstack([np.minimum(b[:3], o[:3]), np.maximum(b[3:], o[3:])])
            box[node] = b
            frm, node = node, parent.get(node, -1)
    return box, used_local


def overlap(a, b):
    return bool(np.all(a[:3] <= b[3:]) and np.all(b[:3] <= a[3:]))


def traverse(child, n, box, leaf, q):
    """k_traverse's walk: children tested at their parent."""
    hits = []

    def nbox(c):
        return leaf[~c] if c < 0 else box[c]

    if not overlap(q, box[0]):
        return hits
    stack, node = [], 0
    while True:
        l, r = child[node]
        ol, orr = overlap(q, nbox(l)), overlap(q, nbox(r))
        if ol and l < 0:
            hits.append(~l)
        if orr and r < 0:
            hits.append(~r)
        dl, dr = ol and l >= 0, orr and r >= 0
        if dl and dr:
            stack.append(r)
            node = l
        elif dl:
            node = l
        elif dr:
            node = r
        elif stack:
            node = stack.pop()
        else:
            return hits


def depth(child):
    best, stack = 0, [(0, 1)]
    while stack:
        c, d = stack.pop()
        best = max(best, d)
        for ch in child[c]:
            if ch >= 0:
                stack.append((ch, d + 1))
    return best


def test_inner_node_index_is_an_end_of_its_range():
    r = np.random.default_rng(11)
    for n, bits in ((2, 30), (3, 30), (257, 30), (1500, 30), (1500, 6)):
        keys = sample_keys(r, n, bits)
        child, rng_ = karras(keys)
        for i, (lo, hi) in enumerate(rng_):
            assert i in (lo, hi)
            l, rr = child[i]
            # the children split the range at gamma
            gl = ~l if l < 0 else rng_[l][1]
            gr = ~rr if rr < 0 else rng_[rr][0]
            assert (l < 0 or rng_[l][0] == lo) and (rr < 0 or rng_[rr][1] == hi)
            assert gr == gl + 1


def test_chunked_refit_equals_plain_refit_in_any_arrival_order():
    r = np.random.default_rng(12)
    for n, bits, chunk in ((1500, 30, 256), (1500, 6, 256), (700, 30, 64), (300, 30, 256)):
        keys = sample_keys(r, n, bits)
        child, rng_ = karras(keys)
        ids = [k & 0xffffffff for k in keys]
        leaf = leaf_boxes(r, n)[ids]                # leaf s = the primitive sorted to slot s
        want = plain_refit(child, n, leaf)
        for trial in range(3):
            order = r.permutation(n)
            got, used_local = chunked_refit(child, rng_, n, leaf, chunk, order)
            assert set(got) == set(want)
            for k in want:
                assert np.array_equal(got[k], want[k])
            assert used_local                       # the lower levels do hand over inside chunks


def test_child_test_walk_finds_exactly_the_overlapping_leaves():
    r = np.random.default_rng(13)
    n = 1200
    keys = sample_keys(r, n, 30)
    child, _ = karras(keys)
    ids = [k & 0xffffffff for k in keys]
    leaf = leaf_boxes(r, n)[ids]
    box = plain_refit(child, n, leaf)
    for _ in range(200):
        lo = r.uniform(-1.2, 1.0, size=3)
        q = np.hstack([lo, lo + r.uniform(0.0, 0.3, size=3)])
        got = sorted(traverse(child, n, box, leaf, q))
        want = [s for s in range(n) if overlap(q, leaf[s])]
        assert got == want


def test_depth_is_within_the_traversal_stack():
    r = np.random.default_rng(14)
    for bits in (30, 8):
        child, _ = karras(sample_keys(r, 4000, bits))
        assert depth(child) < 96


def bitonic_slice_sort(vals):
    """k_sort_query_slices' network for a slice longer than 64: padded with
    INT_MAX to a power of two P >= 128, compare-exchange over (k, j), the
    element pairs (i, i ^ j) ascending where i & k == 0."""
    m = len(vals)
    P = 128
    while P < m:
        P <<= 1
    sh = list(vals) + [0x7fffffff] * (P - m)
    k = 2
    while k <= P:
        j = k >> 1
        while j > 0:
            for i in range(P):
                l = i ^ j
                if l > i:
                    x, y = sh[i], sh[l]
                    if (x > y) if (i & k) == 0 else (x < y):
                        sh[i], sh[l] = y, x
            j >>= 1
        k <<= 1
    return sh[:m]


def test_slice_bitonic_network_sorts_every_length():
    r = np.random.default_rng(15)
    for m in list(range(65, 140)) + [255, 256, 257, 511, 1000, 1023, 1024, 1025, 2047, 2048]:
        vals = r.choice(200000, size=m, replace=False).tolist()   # a slice's primitives are distinct
        assert bitonic_slice_sort(vals) == sorted(vals)
