"""The irregular wave-maker's component sum: the reference's pairwise tree over nleaf = 2^(K-1)
leaves (ColumnSumReduce / RowSumReduce, compute.hlsl:1196-1212; the real components first, the
rest constant sea-level padding) against the warp-split evaluation of the fused kernels (k_boundary: lanes take
aligned parts of the smallest power-of-two range holding the real components, a shuffle tree
joins them, the padding follows).  Both are restated here in float32 arithmetic; the claim under
test is that the regrouping rounds identically, because every padding block sums to an exact
power-of-two multiple of the sea level.
"""
from __future__ import annotations

import numpy as np
import pytest

f32 = np.float32


def tree_range(vals, sea, nreal, m0, m1, carry=None, carry_size=0):
    """Stack form of the pairwise tree over [m0, m1) (vals: (n, 3) float32 leaf triples)."""
    stk, sz = [], []
    if carry_size:
        stk.append(carry)
        sz.append(carry_size)
    m = m0
    while m < m1:
        if m < nreal:
            v, s = vals[m].copy(), 1
        else:
            s = m1 if m == 0 else (m & -m)
            while m + s > m1:
                s >>= 1
            v = np.array([f32(s) * sea, 0, 0], dtype=f32)
        m += s
        stk.append(v)
        sz.append(s)
        while len(sz) >= 2 and sz[-1] == sz[-2]:
            r, l_ = stk.pop(), stk.pop()
            sz.pop()
            stk.append((l_ + r).astype(f32))
            sz[-1] *= 2
    return stk[0]


def warp_split(vals, sea, nreal, nleaf):
    if nreal == 0:
        return tree_range(vals, sea, 0, 0, nleaf)
    R = 1
    while R < nreal:
        R <<= 1
    A = min(32, R)
    per = R // A
    lanes = [tree_range(vals, sea, nreal, k * per, (k + 1) * per) for k in range(A)]
    off = 1
    while off < A:
        lanes = [(lanes[k] + lanes[k + off]).astype(f32) if k % (2 * off) == 0 else lanes[k]
                 for k in range(A - off)] + lanes[A - off:]
        off <<= 1
    v = lanes[0]
    if R < nleaf:
        v = tree_range(vals, sea, nreal, R, nleaf, v, R)
    return v


@pytest.mark.parametrize("nleaf", [1, 2, 8, 64, 256, 2048])
def test_warp_split_matches_the_sequential_tree_bit_for_bit(nleaf):
    rng = np.random.default_rng(nleaf)
    for trial in range(40):
        nreal = int(rng.integers(0, min(nleaf, 300) + 1))
        sea = f32(rng.choice([0.0, 0.37, -1.25, 3.0e3, rng.normal()]))
        vals = np.stack([sea + rng.normal(0, 1, nleaf).astype(f32),
                         rng.normal(0, 2, nleaf).astype(f32),
                         rng.normal(0, 2, nleaf).astype(f32)], axis=1).astype(f32)
        a = tree_range(vals, sea, nreal, 0, nleaf)
        b = warp_split(vals, sea, nreal, nleaf)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (nleaf, nreal, sea, a, b)
