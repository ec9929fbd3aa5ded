"""The treecode build's loop-free pre-order: in a full binary tree a node
over sources [lo, hi) holding L leaves has 2 L - 1 nodes, and its pre-order
index is depth + 2 * (leaves before lo) - (right turns on its path).  The
GPU build computes sizes and indices from that identity (one scan of the
leaves' start flags instead of a pass per level); here it is checked against
an explicit pre-order walk on midpoint-split trees (the reference's split
rule, chebcode.rs:347-388) over random and clustered spectra."""
import bisect

import numpy as np
import pytest


def midpoint_tree(x, leaf_cap, max_depth=48):
    """Nodes as dicts (lo, hi, depth, rturn, left, right), root first."""
    nodes = [dict(lo=0, hi=len(x), depth=0, rturn=0, left=-1, right=-1)]
    stack = [0]
    while stack:
        i = stack.pop()
        nd = nodes[i]
        lo, hi = nd["lo"], nd["hi"]
        if hi - lo <= leaf_cap or nd["depth"] >= max_depth:
            continue
        mid = x[lo] + 0.5 * (x[hi - 1] - x[lo])
        split = bisect.bisect_right(x, mid, lo, hi)
        if split in (lo, hi):
            split = (lo + hi) // 2
        for k, (a, b) in enumerate(((lo, split), (split, hi))):
            nodes.append(dict(lo=a, hi=b, depth=nd["depth"] + 1, rturn=nd["rturn"] + k,
                              left=-1, right=-1))
            nd["left" if k == 0 else "right"] = len(nodes) - 1
            stack.append(len(nodes) - 1)
    return nodes


def preorder(nodes):
    order, sizes = {}, {}

    def walk(i):
        order[i] = len(order)
        n = 1
        if nodes[i]["left"] >= 0:
            n += walk(nodes[i]["left"]) + walk(nodes[i]["right"])
        sizes[i] = n
        return n

    walk(0)
    return order, sizes


@pytest.mark.parametrize("kind,p,leaf_cap", [("uniform", 5000, 32), ("clustered", 3000, 16),
                                             ("spiked", 8000, 11), ("ties", 2000, 8)])
def test_preorder_identity(kind, p, leaf_cap):
    rng = np.random.default_rng(p)
    if kind == "uniform":
        x = rng.random(p)
    elif kind == "clustered":
        x = np.concatenate([rng.normal(0, 1e-3, p // 2), rng.normal(5, 1.0, p - p // 2)])
    elif kind == "spiked":
        x = np.concatenate([rng.random(p - 20), np.exp(rng.uniform(1, 4, 20))])
    else:
        x = np.round(rng.random(p) * 50) / 50  # many equal values
    x = np.sort(x).tolist()
    nodes = midpoint_tree(x, leaf_cap)
    order, sizes = preorder(nodes)
    starts = sorted(nd["lo"] for nd in nodes if nd["left"] < 0)
    for i, nd in enumerate(nodes):
        before = bisect.bisect_left(starts, nd["lo"])
        inside = bisect.bisect_left(starts, nd["hi"]) - before
        assert sizes[i] == 2 * inside - 1
        assert order[i] == nd["depth"] + 2 * before - nd["rturn"]
