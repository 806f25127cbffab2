"""The rule by which the device builds every tree level at once (h2.cu: k_tree_marks,
k_tree_scan, k_tree_emit, k_tree_finish), restated in Python and checked against the oracle's
level-by-level splitting on the CPU: same node table, bit for bit.

With delta_i the number of leading base-2^d digits that sorted keys i-1 and i share (-1 at
i = 0 and at the sentinel i = n), point s starts the nodes of levels f_s = delta_s + 1 .. m_s
when the node of level delta_s around it holds more than leaf_size points; m_s is the first
level whose node starting at s holds at most leaf_size points (capped at the key depth L).
Nodes are numbered level by level in key order; B_l = {starts with f <= l} gives each node's
end (the next entry of B_l), parent (the entry of B_{l-1} at or before it) and children (the
entries of B_{l+1} inside it).
"""
import bisect

import numpy as np
import pytest

import oracle as O


def _tree_from_keys(keys, d, L, leaf):
    n = len(keys)
    keys = [int(k) for k in keys]
    delta = [-1] * (n + 1)
    for i in range(1, n):
        x = keys[i - 1] ^ keys[i]
        delta[i] = L if x == 0 else (64 - x.bit_length() - (64 - d * L)) // d
    fm = [None] * n
    for s in range(n):
        ds, f = delta[s], delta[s] + 1
        E = s == 0
        if s > 0:
            j = s - 1
            while delta[j] >= ds and s - j <= leaf:
                j -= 1
            left = s - j
            if left > leaf:
                E = True
            else:
                k = s + 1
                while k < n and delta[k] >= ds and left + (k - s) <= leaf:
                    k += 1
                E = left + (k - s) > leaf
        if f > L:
            E = False
        if E:
            mu, j, last = L + 1, s + 1, min(s + leaf, n)
            while j <= last and mu >= f:
                mu = min(mu, delta[j])
                j += 1
            fm[s] = (f, min(L, max(f, mu + 1)))
    B = [[] for _ in range(L + 1)]
    at = [[] for _ in range(L + 1)]
    for s in range(n):
        if fm[s] is None:
            continue
        f, m = fm[s]
        for l in range(f, L + 1):
            B[l].append(s)
            if l <= m:
                at[l].append(s)
    begin = np.cumsum([0] + [len(a) for a in at])
    ids = {(l, s): begin[l] + r for l in range(L + 1) for r, s in enumerate(at[l])}
    nn = int(begin[-1])
    out = {k: np.zeros(nn, dtype=np.int32) for k in ("start", "end", "level", "parent", "first_child", "n_child",
                                                     "is_leaf")}
    pos = [{s: i for i, s in enumerate(b)} for b in B]
    for (l, s), t in ids.items():
        f, m = fm[s]
        p = pos[l][s]
        e = B[l][p + 1] if p + 1 < len(B[l]) else n
        out["start"][t], out["end"][t], out["level"][t], out["is_leaf"][t] = s, e, l, int(l == m)
        if l == 0:
            out["parent"][t] = -1
        else:
            br = bisect.bisect_left(B[l - 1], s)
            out["parent"][t] = ids[(l - 1, B[l - 1][br if f <= l - 1 else br - 1])]
        if l < m:
            out["first_child"][t] = ids[(l + 1, s)]
            c0, c = pos[l + 1][s], 0
            while c0 + c < len(B[l + 1]) and B[l + 1][c0 + c] < e:
                c += 1
            out["n_child"][t] = c
        else:
            out["first_child"][t], out["n_child"][t] = -1, 0
    return out


def _cases():
    rng = np.random.default_rng(0)
    Y = rng.normal(size=(2, 1500))
    yield "gaussian 2D", Y, 30
    yield "gaussian 2D, small leaves", Y, 5
    Yc = rng.normal(size=(2, 1200)) * 1e-3 + rng.integers(0, 3, size=(2, 1200))
    yield "clusters 2D", Yc, 25
    Yd = rng.normal(size=(2, 900))
    Yd[:, 200:520] = 0.125
    yield "a block of equal points (depth L)", Yd, 20
    yield "gaussian 3D", rng.normal(size=(3, 1400)), 35
    yield "root is a leaf", rng.normal(size=(2, 40)), 100


@pytest.mark.parametrize("name,Y,leaf", list(_cases()), ids=[c[0] for c in _cases()])
def test_all_levels_rule_equals_level_by_level_splitting(name, Y, leaf):
    h = O.H2(Y, leaf_size=leaf, tol=1e-2)
    d = Y.shape[0]
    ref = h.nodes()
    mine = _tree_from_keys(h.keys(), d, 24 if d == 2 else 20, leaf)
    for k in ref:
        np.testing.assert_array_equal(mine[k], ref[k], err_msg=f"{name}: {k}")
