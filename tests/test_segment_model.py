"""The node-level restatement of the reference's segment walk that the
device's node-parallel walk (begputhinning_b200/csrc/segments.cu,
node_walk_kernel) implements, written as a plain sequential model and
checked against the oracle: chains followed as one step, nodes processed in
any order that respects their raster-earlier graph neighbours (here a FIFO
of ready nodes), +1 on the node a walk ends at, a stall when the exit node
was visited already."""
import collections

import numpy as np

from oracle import pyoracle as po
from tests.helpers import blobs2d, random2d

# 8-neighbour scan order of the reference walk, as (dy, dx)
SCAN = [(-1, -1), (-1, 0), (-1, 1), (0, -1), (0, 1), (1, -1), (1, 0), (1, 1)]
ND = len(SCAN)


def classify(img):
    """2 for points with exactly two point neighbours, -max(n, 1) otherwise,
    0 for background and the outer frame."""
    h, w = img.shape
    v0 = np.zeros((h, w), np.int64)
    for y in range(1, h - 1):
        for x in range(1, w - 1):
            if img[y, x]:
                n = int(img[y - 1:y + 2, x - 1:x + 2].sum()) - 1
                v0[y, x] = 2 if n == 2 else -max(n, 1)
    return v0


def is_end_value(v):
    return -2 < v < 2


def node_model(img):
    """Segments in the reference's emission order, or a string naming the
    rule that did not hold."""
    h, w = img.shape
    v0 = classify(img).ravel()
    off = [dy * w + dx for dy, dx in SCAN]
    nodes = [i for i in range(h * w) if v0[i] < 0]

    # chain pixels: their two neighbours; chain ends: next to a node
    nbrs, ends = {}, set()
    for i in range(h * w):
        if v0[i] != 2:
            continue
        ds = [d for d in range(ND) if v0[i + off[d]] != 0]
        if len(ds) != 2:
            return "chain pixel without two point neighbours"
        nbrs[i] = ds
        if any(v0[i + off[d]] < 0 for d in ds):
            ends.add(i)

    # each end's chain: pixel list to the far end, and the exit scan index
    chain, exit_dir = {}, {}
    for q in ends:
        a, b = nbrs[q]
        if v0[q + off[a]] < 0 and v0[q + off[b]] < 0:
            chain[q], exit_dir[q] = [q], None  # one pixel between two nodes
            continue
        step = a if v0[q + off[a]] == 2 else b
        prev, cur, path = q, q + off[step], [q]
        while True:
            path.append(cur)
            ca, cb = nbrs[cur]
            nxt = cb if cur + off[ca] == prev else ca
            if v0[cur + off[nxt]] < 0:
                chain[q], exit_dir[q] = path, nxt
                break
            prev, cur = cur, cur + off[nxt]

    def exit_of(q, entry_dir):
        if exit_dir[q] is None:
            a, b = nbrs[q]
            back = ND - 1 - entry_dir
            return q + off[b if a == back else a]
        return chain[q][-1] + off[exit_dir[q]]

    def graph_nbr(p, d):
        n = p + off[d]
        if v0[n] < 0:
            return n
        if v0[n] == 2 and n in ends:
            return exit_of(n, d)
        return -1

    indeg = {p: sum(1 for d in range(ND) if 0 <= graph_nbr(p, d) < p) for p in nodes}
    value = {i: int(v0[i]) for i in range(h * w) if v0[i] != 0}
    used = set()
    out = {}
    ready = collections.deque(p for p in nodes if indeg[p] == 0)
    while ready:
        p = ready.popleft()
        budget = -value[p]
        segs = []
        if budget > 0:
            value[p] = 0
            cursor = -1
            for _ in range(budget):
                is_end = is_end_value(v0[p])
                seg = [p]
                nonzero = [d for d in range(cursor + 1, ND) if value.get(p + off[d], 0) != 0]
                cursor = nonzero[0] if nonzero else ND
                if cursor < ND:
                    n = p + off[cursor]
                    if value[n] == 2 and n in ends:
                        if n in used:
                            return "used chain entered again"
                        far = chain[n][-1]
                        e = exit_of(n, cursor)
                        seg += chain[n]
                        used.update((n, far))
                        value[n] = 0
                        if value.get(e, 0) == 0:  # exit visited: the walk stalls on the far end
                            value[far] = 1
                            seg.append(far)
                            is_end |= is_end_value(v0[far])
                        else:
                            value[far] = 0
                            value[e] += 1
                            seg.append(e)
                            is_end |= is_end_value(v0[e])
                    else:
                        if value[n] == 2:
                            return "value-2 point that is not a chain end"
                        value[n] += 1
                        seg.append(n)
                        is_end |= is_end_value(v0[n])
                segs.append((int(is_end), tuple((int(s % w), int(s // w)) for s in seg)))
        out[p] = segs
        for d in range(ND):
            m = graph_nbr(p, d)
            if m > p:
                indeg[m] -= 1
                if indeg[m] == 0:
                    ready.append(m)
    if len(out) != len(nodes):
        return f"{len(nodes) - len(out)} nodes never became ready"
    return [s for p in nodes for s in out[p]]


def test_node_level_model_equals_oracle():
    rng = np.random.default_rng(21)
    cases = []
    for h, w, kind in [(16, 16, "r"), (40, 70, "b"), (64, 64, "r"), (90, 90, "r")]:
        img = blobs2d(rng, h, w, max(1, h * w // 600)) if kind == "b" else random2d(rng, h, w, 0.45)
        cases.append(po.thin2d(img)[0])
    rng2 = np.random.default_rng(22)
    for k in range(3):
        cases.append(random2d(rng2, 40 + 7 * k, 50 + 5 * k, 0.3 + 0.1 * k))
    for k, img in enumerate(cases):
        got = node_model(img)
        assert not isinstance(got, str), f"case {k}: {got}"
        assert got == po.segments2d(img).as_lists(), f"case {k}"
