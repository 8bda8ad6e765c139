"""The size-greedy 4-wide collapse of the build (csrc/gi_kernels.cu:
karras_node in k_karras_leaves, k_state_tables, k_wide_flags, k_collapse),
restated on the CPU: the per-node state tables composed up the parent chain
pick exactly the wide nodes of a top-down greedy expansion (open the part with
the most leaves, ties to the leftmost, twice after the node itself), on radix
trees of uniform, clustered and duplicate sorted keys.  The kernels' own output is covered by the GPU parity
tests; this pins the equivalence the kernels rely on."""
import random

import pytest

LEAF = 1 << 31
W, O2, O3 = 0, 1, 2


def radix_tree(keys):
    """Karras' binary radix tree over sorted 30-bit keys (ties by index):
    child[i] = (left, right, leaves under left, leaves under right)."""
    n = len(keys)

    def delta(i, j):
        if j < 0 or j >= n:
            return -1
        x = keys[i] ^ keys[j]
        return 32 + (32 - (i ^ j).bit_length()) if x == 0 else 32 - x.bit_length()

    child, parent = [None] * (n - 1), [-1] * (n - 1)
    for i in range(n - 1):
        d = 1 if delta(i, i + 1) - delta(i, i - 1) >= 0 else -1
        dmin = delta(i, i - d)
        lmax = 2
        while delta(i, i + lmax * d) > dmin:
            lmax *= 2
        l, t = 0, lmax // 2
        while t >= 1:
            if delta(i, i + (l + t) * d) > dmin:
                l += t
            t //= 2
        j = i + l * d
        dn = delta(i, j)
        s, t = 0, l
        while True:
            t = (t + 1) // 2
            if delta(i, i + (s + t) * d) > dn:
                s += t
            if t <= 1:
                break
        g = i + s * d + min(d, 0)
        lo, hi = min(i, j), max(i, j)
        left = (LEAF | g) if lo == g else g
        right = (LEAF | (g + 1)) if hi == g + 1 else g + 1
        child[i] = (left, right, g - lo + 1, hi - g)
        for c in (left, right):
            if not c & LEAF:
                parent[c] = i
    return child, parent


def expand(child, r):
    """Parts of wide node r: open r, then twice the largest internal part."""
    c = child[r]
    slot, num = [c[0], c[1]], [c[2], c[3]]
    for _ in range(2):
        b = max(range(len(num)), key=lambda k: (num[k], -k))
        if num[b] < 2:
            break
        g = child[slot[b]]
        slot[b:b + 1] = [g[0], g[1]]
        num[b:b + 1] = [g[2], g[3]]
    return slot


def first_max3(a, b, c):
    k, m = 0, a
    if b > m:
        k, m = 1, b
    if c > m:
        k = 2
    return k


def state_table(child, parent, y):
    p = parent[y]
    c = child[p]
    left = c[0] == y
    z = c[1] if left else c[0]
    ny, nz = (c[2], c[3]) if left else (c[3], c[2])
    if (ny >= nz) if left else (ny > nz):
        sw = O2
    else:
        g = child[z]
        sw = O3 if (first_max3(ny, g[2], g[3]) == 0 if left else first_max3(g[2], g[3], ny) == 2) else W
    so2 = W
    r = parent[p]
    if r >= 0:
        cr = child[r]
        pleft = cr[0] == p
        ns = cr[3] if pleft else cr[2]
        mine = (0 if left else 1) if pleft else (1 if left else 2)
        k = first_max3(c[2], c[3], ns) if pleft else first_max3(ns, c[2], c[3])
        so2 = O3 if k == mine else W
    return (sw, so2, W)


def wide_flags(child, parent):
    n1 = len(child)
    tab = [None] + [state_table(child, parent, y) for y in range(1, n1)]
    flags = [True] + [False] * (n1 - 1)
    for i in range(1, n1):
        f, x = tab[i], parent[i]
        while x > 0 and not (f[0] == f[1] == f[2]):
            f = tuple(f[s] for s in tab[x])
            x = parent[x]
        flags[i] = f[0] == W
    return flags


def top_down(child):
    wide, stack = {0}, [0]
    while stack:
        for c in expand(child, stack.pop()):
            if not c & LEAF:
                wide.add(c)
                stack.append(c)
    return wide


def _keys(rng, kind, n):
    if kind == "uniform":
        ks = [rng.getrandbits(30) for _ in range(n)]
    elif kind == "clustered":  # few distinct prefixes, long shared runs: uneven splits
        ks = [(rng.choice([0x0F0F0F0, 0x2AAAAAA, 0x3FFFF00]) ^ rng.getrandbits(rng.choice([2, 6, 12]))) for _ in range(n)]
    else:  # many exact duplicates: the tie-break by index decides the splits
        ks = [rng.getrandbits(4) << 26 for _ in range(n)]
    return sorted(ks)


@pytest.mark.parametrize("kind", ["uniform", "clustered", "duplicates"])
@pytest.mark.parametrize("n", [2, 3, 5, 17, 1000, 2500])
def test_state_tables_match_top_down_greedy(kind, n):
    rng = random.Random(n * 7 + len(kind))
    child, parent = radix_tree(_keys(rng, kind, n))
    flags = wide_flags(child, parent)
    want = top_down(child)
    assert {i for i, f in enumerate(flags) if f} == want
    # every leaf sits in exactly one slot of one wide node; every wide node but the root in one slot
    seen = [0] * n
    up = {0: 1}
    for w in want:
        parts = expand(child, w)
        assert 2 <= len(parts) <= 4 and all((p & LEAF) or p in want for p in parts)
        for p in parts:
            if p & LEAF:
                seen[p & ~LEAF] += 1
            else:
                up[p] = up.get(p, 0) + 1
    assert seen == [1] * n and all(v == 1 for v in up.values()) and len(up) == len(want)
