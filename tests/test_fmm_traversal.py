"""The dual-tree traversal the GPU runs level by level without reading its
sizes back, restated in numpy and checked on the CPU.

The traversal (fast-multipole.cc:484-526, `fmm_traverse_kernel`) starts from
(root, root); a pair is accepted for M2L when (r_t + r_s)^2 < theta^2 d^2,
kept for P2P when both cells are leaves, and otherwise split on the source
when it is the only non-leaf or has the larger radius, on the target
otherwise. Splitting one cell raises the pair's depth sum by one, so every
pair of level L has depth sum L and the traversal ends after at most
2 max_depth + 1 levels: the bound the GPU uses to launch its levels without
a read-back. The lists cover every ordered particle pair exactly once."""
import numpy as np
import pytest


def build_tree(pts, cap):
    """Octree over the cube bounding the points; cells with more than cap
    points split into their non-empty octants. Points are reordered so that
    each cell is a contiguous range. Returns (order, nodes) with nodes as
    dicts {lo, hi, centre, radius, depth, children}."""
    lo, hi = pts.min(axis=0), pts.max(axis=0)
    centre = 0.5 * (lo + hi)
    half = 0.5 * float(np.max(hi - lo)) * (1 + 1e-12)
    nodes, order = [], []

    def make(idx, c, h, depth):
        k = len(nodes)
        node = {"centre": c, "depth": depth, "children": [], "lo": len(order)}
        nodes.append(node)
        if len(idx) <= cap:
            order.extend(idx.tolist())
        else:
            rel = pts[idx] >= c
            octant = rel[:, 0] * 1 + rel[:, 1] * 2 + rel[:, 2] * 4
            for o in range(8):
                sub = idx[octant == o]
                if len(sub) == 0:
                    continue
                off = np.array([1.0 if (o >> d) & 1 else -1.0 for d in range(3)])
                node["children"].append(make(sub, c + 0.5 * h * off, 0.5 * h, depth + 1))
        node["hi"] = len(order)
        members = pts[order[node["lo"]:node["hi"]]]
        node["radius"] = float(np.sqrt(((members - c) ** 2).sum(axis=1).max()))
        return k

    make(np.arange(len(pts)), centre, half, 0)
    return np.array(order), nodes


def traverse(nodes, theta):
    """Breadth-first dual traversal; returns (m2l, p2p, depth sums per level)."""
    m2l, p2p, levels = [], [], []
    cur = [(0, 0)]
    while cur:
        levels.append({nodes[t]["depth"] + nodes[s]["depth"] for t, s in cur})
        nxt = []
        for t, s in cur:
            T, S = nodes[t], nodes[s]
            d2 = float(((T["centre"] - S["centre"]) ** 2).sum())
            rsum = T["radius"] + S["radius"]
            if rsum * rsum < theta * theta * d2:
                m2l.append((t, s))
                continue
            tleaf, sleaf = not T["children"], not S["children"]
            if tleaf and sleaf:
                p2p.append((t, s))
                continue
            split_target = sleaf or (not tleaf and T["radius"] >= S["radius"])
            if split_target:
                nxt.extend((c, s) for c in T["children"])
            else:
                nxt.extend((t, c) for c in S["children"])
        cur = nxt
    return m2l, p2p, levels


@pytest.mark.parametrize("cap,theta", [(8, 0.5), (16, 0.525), (32, 0.6)])
def test_traversal_levels_and_coverage(cap, theta):
    rng = np.random.default_rng(cap)
    n = 700
    pts = rng.normal(size=(n, 3)) * np.array([1.0, 1.0, 3.0])
    order, nodes = build_tree(pts, cap)
    max_depth = max(nd["depth"] for nd in nodes)
    m2l, p2p, levels = traverse(nodes, theta)
    # level L holds pairs of depth sum L only, and there are at most 2 max_depth + 1 levels
    assert all(lv == {L} for L, lv in enumerate(levels))
    assert len(levels) <= 2 * max_depth + 1
    # every ordered particle pair (the particle with itself included) is covered exactly once
    cover = np.zeros((n, n), dtype=np.int32)
    for t, s in m2l + p2p:
        T, S = nodes[t], nodes[s]
        cover[T["lo"]:T["hi"], S["lo"]:S["hi"]] += 1
    assert np.all(cover == 1)
    # P2P pairs are leaf pairs, M2L pairs are separated by the opening test
    assert all(not nodes[t]["children"] and not nodes[s]["children"] for t, s in p2p)
    assert len(m2l) > 0 and len(p2p) > 0


def test_capacity_overflow_keeps_a_written_prefix():
    # the GPU level writes every child slot below its capacity (reservations
    # are contiguous) and flags the rest: the entries it keeps are exactly
    # the prefix of the full emission order, so a retry with larger lists
    # reproduces the same traversal
    rng = np.random.default_rng(3)
    reserved = np.cumsum(rng.integers(0, 9, size=200))  # per-warp reservation ends
    starts = np.concatenate([[0], reserved[:-1]])
    cap = int(reserved[-1] * 0.6)
    written = np.zeros(reserved[-1], dtype=bool)
    overflow = False
    for b, e in zip(starts, reserved):
        for slot in range(b, e):
            if slot < cap:
                written[slot] = True
            else:
                overflow = True
    assert overflow and written[:cap].all() and not written[cap:].any()
