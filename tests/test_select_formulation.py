"""The data-parallel form of libstdc++'s introselect / introsort used by the
top-k kernel (nexdynipc_b200/csrc/select.cuh), restated in Python step for
step, against std::nth_element + std::sort run by the oracle library.

The GPU test tests/test_gpu_parity.py checks the device kernel itself on the
same kind of inputs; this test pins the formulation (the G/L partition
identity and the stable finishing sort) on many more cases.
"""
import numpy as np
import pytest

from oracle import refcpu


def lg(n):
    return n.bit_length() - 1


class Sel:
    def __init__(self, keys):
        self.k = np.asarray(keys, dtype=np.float64)
        self.idx = list(range(len(keys)))

    def less(self, a, b):
        return self.k[a] < self.k[b]

    def median_to_first(self, r, a, b, c):
        I = self.idx
        if self.less(I[a], I[b]):
            if self.less(I[b], I[c]): sw = b
            elif self.less(I[a], I[c]): sw = c
            else: sw = a
        elif self.less(I[a], I[c]): sw = a
        elif self.less(I[b], I[c]): sw = c
        else: sw = b
        I[r], I[sw] = I[sw], I[r]

    def partition(self, first, last):
        # G/L formulation of __unguarded_partition (pivot at `first`)
        I, K = self.idx, self.k
        pk = K[I[first]]
        G = [p for p in range(first + 1, last) if not (K[I[p]] < pk)]
        L = [p for p in range(last - 1, first - 1, -1) if not (pk < K[I[p]])]
        nswap = sum(1 for t in range(min(len(G), len(L))) if G[t] < L[t])
        for t in range(nswap):
            I[G[t]], I[L[t]] = I[L[t]], I[G[t]]
        gm = G[nswap] if nswap < len(G) else 1 << 40
        lm = L[nswap - 1] if nswap >= 1 else 1 << 40
        return min(gm, lm)

    def partition_pivot(self, first, last):
        mid = first + (last - first) // 2
        self.median_to_first(first, first + 1, mid, last - 1)
        return self.partition(first, last)

    def insertion_sort(self, first, last):
        I = self.idx
        for i in range(first + 1, last):
            v = I[i]
            if self.less(v, I[first]):
                I[first + 1:i + 1] = I[first:i]
                I[first] = v
            else:
                j = i
                while self.less(v, I[j - 1]):
                    I[j] = I[j - 1]
                    j -= 1
                I[j] = v

    def adjust_heap(self, first, hole, ln, value):
        I = self.idx
        top = hole
        second = hole
        while second < (ln - 1) // 2:
            second = 2 * (second + 1)
            if self.less(I[first + second], I[first + second - 1]):
                second -= 1
            I[first + hole] = I[first + second]
            hole = second
        if (ln & 1) == 0 and second == (ln - 2) // 2:
            second = 2 * (second + 1)
            I[first + hole] = I[first + second - 1]
            hole = second - 1
        parent = (hole - 1) // 2 if hole > 0 else 0
        while hole > top and self.less(I[first + parent], value):
            I[first + hole] = I[first + parent]
            hole = parent
            parent = (hole - 1) // 2 if hole > 0 else 0
        I[first + hole] = value

    def make_heap(self, first, last):
        ln = last - first
        if ln < 2:
            return
        parent = (ln - 2) // 2
        while True:
            self.adjust_heap(first, parent, ln, self.idx[first + parent])
            if parent == 0:
                return
            parent -= 1

    def pop_heap(self, first, last, result):
        v = self.idx[result]
        self.idx[result] = self.idx[first]
        self.adjust_heap(first, 0, last - first, v)

    def heap_select(self, first, middle, last):
        self.make_heap(first, middle)
        for i in range(middle, last):
            if self.less(self.idx[i], self.idx[first]):
                self.pop_heap(first, middle, i)

    def nth_element(self, n, nth):
        first, last = 0, n
        depth = lg(n) * 2
        while last - first > 3:
            if depth == 0:
                self.heap_select(first, nth + 1, last)
                self.idx[first], self.idx[nth] = self.idx[nth], self.idx[first]
                return
            depth -= 1
            cut = self.partition_pivot(first, last)
            if cut <= nth:
                first = cut
            else:
                last = cut
        self.insertion_sort(first, last)

    def sort_small(self, k):
        if k <= 1:
            return
        if k > 16:
            stack = [(0, k, lg(k) * 2)]
            while stack:
                f, l, d = stack.pop()
                while l - f > 16:
                    if d == 0:
                        self.heap_select(f, l, l)
                        while l - f > 1:
                            l -= 1
                            self.pop_heap(f, l, l)
                        break
                    d -= 1
                    cut = self.partition_pivot(f, l)
                    stack.append((cut, l, d))
                    l = cut
        head = self.idx[:k]
        ranks = []
        for a, e in enumerate(head):
            r = sum(1 for b, o in enumerate(head) if self.k[o] < self.k[e] or (self.k[o] == self.k[e] and b < a))
            ranks.append(r)
        out = [0] * k
        for e, r in zip(head, ranks):
            out[r] = e
        self.idx[:k] = out

    def top_k(self, k):
        n = len(self.idx)
        if k < n:
            self.nth_element(n, k)
        self.sort_small(k)
        return self.idx[:k]


def cases():
    rng = np.random.default_rng(7)
    out = []
    for n in (1, 2, 3, 4, 5, 16, 17, 31, 32, 33, 40, 64, 100, 124, 186, 642, 1920):
        out.append(np.zeros(n))                                   # all ties
        out.append(rng.integers(0, 3, n).astype(float))           # heavy ties
        out.append(rng.random(n))                                  # distinct
        z = rng.random(n); z[rng.random(n) < 0.6] = 0.0            # zeros + values
        out.append(z)
        out.append(np.arange(n, dtype=float)[::-1].copy())         # descending
        out.append(np.sort(rng.random(n)))                         # ascending
    return out


@pytest.mark.parametrize("keys", cases(), ids=lambda k: f"n{len(k)}")
def test_formulation_matches_libstdcxx(keys):
    k = min(32, len(keys))
    expect = refcpu.select_top_k(keys, k).tolist()
    got = Sel(keys).top_k(k)
    assert got == expect


def test_std_sort_stable_rank_finish():
    # std::sort of <= 16 elements is the stable insertion sort of the input
    rng = np.random.default_rng(3)
    for _ in range(200):
        n = int(rng.integers(1, 17))
        keys = rng.integers(0, 4, n).astype(float)
        got = refcpu.std_sort(keys).tolist()
        assert got == sorted(range(n), key=lambda i: (keys[i], i))


# ---------------------------------------------------------------------------
# The contact sort (sel_sort_prefix_block): std::sort of the raw contacts by
# distance, exact in the first `keep` positions, formulated as CTA-partitioned
# long ranges, warp-finished short ranges, leaves stably sorted, and ranges
# that start at or beyond `keep` dropped.
# ---------------------------------------------------------------------------
def sort_heap(s, f, l):
    while l - f > 1:
        l -= 1
        s.pop_heap(f, l, l)


def finish_range(s, f, l, d, keep):
    """One warp's range: introsort with leaves marked, then the stable sort
    of each leaf."""
    leaves = []
    stack = [(f, l, d)]
    while stack:
        a, b, dd = stack.pop()
        while True:
            if a >= keep or b - a <= 16:
                break
            if dd == 0:
                s.make_heap(a, b)
                sort_heap(s, a, b)
                break
            dd -= 1
            cut = s.partition_pivot(a, b)
            stack.append((cut, b, dd))
            b = cut
        leaves.append(a)
    starts = sorted(leaves) + [l]
    for a, b in zip(starts[:-1], starts[1:]):
        s.idx[a:b] = sorted(s.idx[a:b], key=lambda e, pos={e: p for p, e in enumerate(s.idx[a:b])}: (s.k[e], pos[e]))


def sort_prefix(keys, keep, warp_range=256):
    s = Sel(keys)
    n = len(keys)
    small = []
    stack = [(0, n, 2 * lg(n))]
    while stack:
        f, l, d = stack.pop()
        while True:
            if f >= keep or l - f <= 1:
                break
            if l - f <= warp_range:
                small.append((f, l, d))
                break
            if d == 0:
                s.make_heap(f, l)
                sort_heap(s, f, l)
                break
            d -= 1
            cut = s.partition_pivot(f, l)
            stack.append((cut, l, d))
            l = cut
    for f, l, d in small:
        finish_range(s, f, l, d, keep)
    return s.idx[:keep]


def contact_like_cases():
    rng = np.random.default_rng(11)
    out = []
    for n, keep in ((2001, 2000), (2600, 2000), (5000, 2000), (9000, 2000), (700, 300), (300, 40)):
        z = rng.random(n) * 1e-3
        z[rng.random(n) < 0.3] = 0.0                      # touching hinged links: distance 0
        z[rng.random(n) < 0.1] = 2.1127e-4                 # a repeated value
        out.append((z, keep))
        out.append((np.round(rng.random(n) * 8) / 8, keep))   # few distinct values
        out.append((np.zeros(n), keep))                      # all equal
        out.append((np.arange(n, dtype=float)[::-1].copy(), keep))
    return out


@pytest.mark.parametrize("case", contact_like_cases(), ids=lambda c: f"n{len(c[0])}_keep{c[1]}")
def test_contact_sort_prefix_matches_std_sort(case):
    keys, keep = case
    expect = refcpu.std_sort(keys).tolist()[:keep]
    assert sort_prefix(keys, keep) == expect
